/* culip's libs/utils/defines.h (namespaces, index types, timers), provided by culip_la.hpp over the culipx C ABI. */
#pragma once
#include <culip_la.hpp>
