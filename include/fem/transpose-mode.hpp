#pragma once

namespace fem {

// Direction of a linear map (include/transpose-mode.hpp:13): NoTranspose
// (nodes -> points, gather) or Transpose (points -> nodes, scatter-add).
enum class ContractMode { NoTranspose, Transpose };

}  // namespace fem
