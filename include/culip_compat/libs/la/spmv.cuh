/* culip's libs/la/spmv.cuh (SPMV<T>, CSRMatrixSPMV<T>), provided by culip_la.hpp over the culipx C ABI. */
#pragma once
#include <culip_la.hpp>
