// Stand-in for the reference's util/assert.hpp (see stub/util/types.hpp):
// the known-answer driver compiles the reference's sfcurves.hpp, whose
// part_by_two21/10 assert their input range; inputs here are in range.
#pragma once
#define mAssert(cond) ((void)0)
