/* culip's libs/la/iterative_solvers/sqmr.cuh (SQMR<T>), provided by culip_la.hpp over the culipx C ABI. */
#pragma once
#include <culip_la.hpp>
