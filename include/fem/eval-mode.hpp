#pragma once

namespace fem {

// What a basis computes and what a QFunction field expects at quadrature
// points (values as the reference's include/eval-mode.hpp:11):
//   None    the field passes through unchanged (e.g. qdata)
//   Interp  values at the quadrature points
//   Grad    reference-space gradients at the quadrature points
//   Weight  quadrature weights (no input vector)
enum class EvalMode { None, Interp, Grad, Weight };

}  // namespace fem
