/* culip's libs/test/test.h (Test<T>, Matrix Market I/O), provided by culip_la.hpp over the culipx C ABI. */
#pragma once
#include <culip_la.hpp>
