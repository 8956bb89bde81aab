/* culip's libs/utils/types.cuh (dense_vector_t, csr_matrix_t, gpu_handle_t), provided by culip_la.hpp over the culipx C ABI. */
#pragma once
#include <culip_la.hpp>
