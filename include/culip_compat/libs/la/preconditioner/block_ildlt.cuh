/* culip's libs/la/preconditioner/block_ildlt.cuh (BlockiLDLt<T, BK, Rook>), provided by culip_la.hpp over the culipx C ABI. */
#pragma once
#include <culip_la.hpp>
