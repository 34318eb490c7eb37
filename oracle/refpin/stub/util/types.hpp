// Stand-in for the reference's util/types.hpp, only for compiling its
// integer headers core/math/rng.hpp and core/math/sfcurves.hpp with g++ to
// produce known answers (oracle/refpin/refpin.cpp). Test infrastructure: the
// real header pulls in the Epsilon vector library, which is absent; rng.hpp
// and sfcurves.hpp need only the integer typedefs (the reference's
// util/int_types.hpp names), the CUDA qualifiers and one vector type of an
// unused Xoroshiro128 member.
#pragma once

#include <cstdint>

#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif

namespace mufflon {
using u8 = std::uint8_t;
using u16 = std::uint16_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;
using i32 = std::int32_t;
} // namespace mufflon

namespace ei {
struct UVec4 { std::uint32_t x, y, z, w; };
} // namespace ei
