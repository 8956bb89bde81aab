/* culip's libs/utils/mem_pool.cuh (GlobalMemPool), provided by culip_la.hpp over the culipx C ABI. */
#pragma once
#include <culip_la.hpp>
