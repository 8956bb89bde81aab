/* culip's libs/la/dense_la.cuh (T_nrm2, T_doti, T_scal, T_axpy), provided by culip_la.hpp over the culipx C ABI. */
#pragma once
#include <culip_la.hpp>
