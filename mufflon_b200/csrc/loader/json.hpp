// A small JSON document model for scene description files.
//
// Objects keep their members in file order (the first scenario of a file is
// its default when none is named, json_loader.cpp load_file). Numbers are
// parsed with std::from_chars (correctly rounded, independent of the C
// locale). Errors carry the line and column of the offending character.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace mffl {

struct JsonError : std::runtime_error { using std::runtime_error::runtime_error; };

struct JsonValue {
	enum Type { NUL, BOOL, NUMBER, STRING, ARRAY, OBJECT };
	Type type = NUL;
	bool boolean = false;
	double number = 0.0;
	std::string string;
	std::vector<JsonValue> array;
	std::vector<std::pair<std::string, JsonValue>> members;

	bool is_null() const { return type == NUL; }
	bool is_bool() const { return type == BOOL; }
	bool is_number() const { return type == NUMBER; }
	bool is_string() const { return type == STRING; }
	bool is_array() const { return type == ARRAY; }
	bool is_object() const { return type == OBJECT; }
	// Member lookup (the last one wins for duplicated keys); nullptr if absent.
	const JsonValue* find(const std::string& key) const;
	JsonValue* find(const std::string& key);
	// Adds or replaces a member.
	void set(const std::string& key, JsonValue value);
};

const char* type_name(JsonValue::Type t);

// Parses a complete document; throws JsonError.
JsonValue parse_json(const std::string& text);

} // namespace mffl
