#include "json.hpp"

#include <charconv>
#include <cstring>

namespace mffl {

const JsonValue* JsonValue::find(const std::string& key) const {
	for(size_t i = members.size(); i-- > 0;)
		if(members[i].first == key) return &members[i].second;
	return nullptr;
}

JsonValue* JsonValue::find(const std::string& key) {
	for(size_t i = members.size(); i-- > 0;)
		if(members[i].first == key) return &members[i].second;
	return nullptr;
}

void JsonValue::set(const std::string& key, JsonValue value) {
	if(JsonValue* v = find(key)) *v = std::move(value);
	else members.emplace_back(key, std::move(value));
}

const char* type_name(JsonValue::Type t) {
	switch(t) {
		case JsonValue::NUL: return "null";
		case JsonValue::BOOL: return "bool";
		case JsonValue::NUMBER: return "number";
		case JsonValue::STRING: return "string";
		case JsonValue::ARRAY: return "array";
		case JsonValue::OBJECT: return "object";
	}
	return "?";
}

namespace {

constexpr int MAX_DEPTH = 256;

class Parser {
public:
	explicit Parser(const std::string& t) : m_t(t) {}

	JsonValue document() {
		JsonValue v = value(0);
		skip_ws();
		if(m_p != m_t.size()) fail("unexpected characters after the document");
		return v;
	}

private:
	const std::string& m_t;
	size_t m_p = 0;

	[[noreturn]] void fail(const std::string& what) const {
		size_t line = 1, col = 1;
		for(size_t i = 0; i < m_p && i < m_t.size(); ++i) {
			if(m_t[i] == '\n') { ++line; col = 1; }
			else ++col;
		}
		throw JsonError("JSON parse error: " + what + " (line " + std::to_string(line) + ", column "
		                + std::to_string(col) + ")");
	}

	void skip_ws() {
		while(m_p < m_t.size()) {
			const char c = m_t[m_p];
			if(c == ' ' || c == '\t' || c == '\n' || c == '\r') ++m_p;
			else break;
		}
	}

	bool literal(const char* word) {
		const size_t n = std::strlen(word);
		if(m_t.compare(m_p, n, word) == 0) { m_p += n; return true; }
		return false;
	}

	JsonValue value(int depth) {
		if(depth > MAX_DEPTH) fail("nesting too deep");
		skip_ws();
		if(m_p >= m_t.size()) fail("unexpected end of input");
		JsonValue v;
		const char c = m_t[m_p];
		if(c == '{') {
			v.type = JsonValue::OBJECT;
			++m_p;
			skip_ws();
			if(m_p < m_t.size() && m_t[m_p] == '}') { ++m_p; return v; }
			for(;;) {
				skip_ws();
				if(m_p >= m_t.size() || m_t[m_p] != '"') fail("expected a member name");
				std::string key = string();
				skip_ws();
				if(m_p >= m_t.size() || m_t[m_p] != ':') fail("expected ':'");
				++m_p;
				v.members.emplace_back(std::move(key), value(depth + 1));
				skip_ws();
				if(m_p >= m_t.size()) fail("unexpected end of input");
				if(m_p < m_t.size() && m_t[m_p] == ',') { ++m_p; continue; }
				if(m_p < m_t.size() && m_t[m_p] == '}') { ++m_p; return v; }
				fail("expected ',' or '}'");
			}
		}
		if(c == '[') {
			v.type = JsonValue::ARRAY;
			++m_p;
			skip_ws();
			if(m_p < m_t.size() && m_t[m_p] == ']') { ++m_p; return v; }
			for(;;) {
				v.array.push_back(value(depth + 1));
				skip_ws();
				if(m_p >= m_t.size()) fail("unexpected end of input");
				if(m_p < m_t.size() && m_t[m_p] == ',') { ++m_p; continue; }
				if(m_p < m_t.size() && m_t[m_p] == ']') { ++m_p; return v; }
				fail("expected ',' or ']'");
			}
		}
		if(c == '"') { v.type = JsonValue::STRING; v.string = string(); return v; }
		if(literal("true")) { v.type = JsonValue::BOOL; v.boolean = true; return v; }
		if(literal("false")) { v.type = JsonValue::BOOL; v.boolean = false; return v; }
		if(literal("null")) return v;
		if(c == '-' || (c >= '0' && c <= '9')) { v.type = JsonValue::NUMBER; v.number = number(); return v; }
		fail(std::string("unexpected character '") + c + "'");
	}

	double number() {
		const size_t start = m_p;
		if(m_t[m_p] == '-') ++m_p;
		auto digits = [&]() {
			const size_t s = m_p;
			while(m_p < m_t.size() && m_t[m_p] >= '0' && m_t[m_p] <= '9') ++m_p;
			return m_p - s;
		};
		if(m_p < m_t.size() && m_t[m_p] == '0') ++m_p;
		else if(digits() == 0) fail("invalid number");
		if(m_p < m_t.size() && m_t[m_p] == '.') { ++m_p; if(digits() == 0) fail("invalid number"); }
		if(m_p < m_t.size() && (m_t[m_p] == 'e' || m_t[m_p] == 'E')) {
			++m_p;
			if(m_p < m_t.size() && (m_t[m_p] == '+' || m_t[m_p] == '-')) ++m_p;
			if(digits() == 0) fail("invalid number");
		}
		double d = 0.0;
		const auto r = std::from_chars(m_t.data() + start, m_t.data() + m_p, d);
		if(r.ec != std::errc() || r.ptr != m_t.data() + m_p) fail("number out of range");
		return d;
	}

	static void put_utf8(std::string& out, uint32_t cp) {
		if(cp < 0x80) out += char(cp);
		else if(cp < 0x800) { out += char(0xC0 | (cp >> 6)); out += char(0x80 | (cp & 0x3F)); }
		else if(cp < 0x10000) {
			out += char(0xE0 | (cp >> 12)); out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F));
		} else {
			out += char(0xF0 | (cp >> 18)); out += char(0x80 | ((cp >> 12) & 0x3F));
			out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F));
		}
	}

	uint32_t hex4() {
		if(m_p + 4 > m_t.size()) fail("truncated \\u escape");
		uint32_t v = 0;
		for(int i = 0; i < 4; ++i) {
			const char c = m_t[m_p++];
			v <<= 4;
			if(c >= '0' && c <= '9') v |= uint32_t(c - '0');
			else if(c >= 'a' && c <= 'f') v |= uint32_t(c - 'a' + 10);
			else if(c >= 'A' && c <= 'F') v |= uint32_t(c - 'A' + 10);
			else fail("invalid \\u escape");
		}
		return v;
	}

	std::string string() {
		++m_p; // opening quote
		std::string out;
		for(;;) {
			if(m_p >= m_t.size()) fail("unterminated string");
			const char c = m_t[m_p++];
			if(c == '"') return out;
			if(static_cast<unsigned char>(c) < 0x20) fail("control character in string");
			if(c != '\\') { out += c; continue; }
			if(m_p >= m_t.size()) fail("unterminated escape");
			const char e = m_t[m_p++];
			switch(e) {
				case '"': out += '"'; break;
				case '\\': out += '\\'; break;
				case '/': out += '/'; break;
				case 'b': out += '\b'; break;
				case 'f': out += '\f'; break;
				case 'n': out += '\n'; break;
				case 'r': out += '\r'; break;
				case 't': out += '\t'; break;
				case 'u': {
					uint32_t cp = hex4();
					if(cp >= 0xD800 && cp < 0xDC00) {
						if(m_p + 2 > m_t.size() || m_t[m_p] != '\\' || m_t[m_p + 1] != 'u') fail("unpaired surrogate");
						m_p += 2;
						const uint32_t lo = hex4();
						if(lo < 0xDC00 || lo >= 0xE000) fail("invalid surrogate pair");
						cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
					} else if(cp >= 0xDC00 && cp < 0xE000) fail("unpaired surrogate");
					put_utf8(out, cp);
					break;
				}
				default: fail(std::string("invalid escape '\\") + e + "'");
			}
		}
	}
};

} // namespace

JsonValue parse_json(const std::string& text) {
	return Parser(text).document();
}

} // namespace mffl
