// Storage of the Rys coefficient table (one copy in the library) and its
// device address for the kernels.
#include "bqc.h"

#define RYS_CONST static __device__ const __align__(16)
#define RYS_CONST_SMALL static const
#include "rys_tables.inc"
#undef RYS_CONST
#undef RYS_CONST_SMALL

const double *bqc_rys_table() {
    // the symbol's device address differs per device; look it up each time
    // (a cheap runtime call) so multi-device processes stay correct
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, RYS_TABLE) != cudaSuccess) return nullptr;
    return static_cast<const double *>(ptr);
}

const double *bqc_rys_table_lm() {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, RYS_TABLE_LM) != cudaSuccess) return nullptr;
    return static_cast<const double *>(ptr);
}
