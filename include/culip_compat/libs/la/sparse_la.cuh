/* culip's libs/la/sparse_la.cuh (T_csrmv, T_matrix_permute_scale), provided by culip_la.hpp over the culipx C ABI. */
#pragma once
#include <culip_la.hpp>
