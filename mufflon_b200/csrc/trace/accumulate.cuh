// Per-iteration accumulation of render targets on the device, as
// output_handler_variance.hpp:7-31 of the reference does it for one channel:
//   * update_moments (UpdateIter<T, false>): the running mean, and, when the
//     target's variance is recorded, its running variance;
//   * update_reduced (UpdateIter<T, true>, targets that reduce moments, e.g.
//     the light tracer's Density, render_targets.hpp:68-74): the iteration's
//     value, and, when the variance slot is recorded, the running mean in it.
// `iteration` is 0 for the first iteration after a reset. Divisions are
// correctly rounded and nothing is contracted, so the CPU oracle's
// restatement produces the same bits.
#pragma once

#include "dmath.cuh"

namespace mb {

MBD void update_moments(float iter, float* cum, float* var, int iteration) {
	const float it = float(iteration);
	const float diff = __fsub_rn(iter, *cum);
	const float c = __fadd_rn(*cum, __fdiv_rn(diff, fmaxf(1.0f, __fadd_rn(it, 1.0f))));
	*cum = c;
	if(var) {
		const float v = *var;
		const float varIter = __fmul_rn(diff, __fsub_rn(iter, c));
		*var = __fadd_rn(v, __fdiv_rn(__fsub_rn(varIter, v), fmaxf(1.0f, it)));
	}
}

MBD void update_reduced(float iter, float* cum, float* mean, int iteration) {
	*cum = iter;
	if(mean) {
		const float m = *mean;
		*mean = __fadd_rn(m, __fdiv_rn(__fsub_rn(iter, m), fmaxf(1.0f, __fadd_rn(float(iteration), 1.0f))));
	}
}

} // namespace mb
