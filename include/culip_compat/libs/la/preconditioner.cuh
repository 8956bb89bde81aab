/* culip's libs/la/preconditioner.cuh (Preconditioner<T>), provided by culip_la.hpp over the culipx C ABI. */
#pragma once
#include <culip_la.hpp>
