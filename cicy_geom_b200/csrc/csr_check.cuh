// Structure check of a caller's CSR system and its chain partition, run once
// on the device before kernels that trust them (column indices used as
// addresses, chains walked row by row).  Flags: 1 row_ptr is not 0 .. nnz
// non-decreasing, 2 a column index is outside [0, n), 4 the chains are not
// consecutive runs of at least one row covering 0 .. n-1.  Every read stays
// within the stated sizes n + 1, nnz and nchains.
#pragma once

#include <cstdint>
#include <string>

namespace cicy {

// This thread's share of the flags, threads t, t + stride, ... of `stride`.
__device__ inline int check_structure_part(int t, int stride, int n, int nnz, const int32_t* rp, const int32_t* ci, int nchains,
                                           const int32_t* cs, const int32_t* cl) {
    int f = 0;
    if (t == 0 && (rp[0] != 0 || rp[n] != nnz)) f |= 1;
    for (int i = t; i < n; i += stride)
        if (rp[i] > rp[i + 1]) f |= 1;
    for (int k = t; k < nnz; k += stride)
        if (ci[k] < 0 || ci[k] >= n) f |= 2;
    for (int c = t; c < nchains; c += stride) {
        const int st = cs[c], ln = cl[c];
        const int expect = c == 0 ? 0 : cs[c - 1] + cl[c - 1];
        if (ln < 1 || st != expect || (c == nchains - 1 && st + ln != n)) f |= 4;
    }
    return f;
}

inline std::string structure_error(int flags) {
    return (flags & 1) ? "row_ptr is not 0 .. nnz non-decreasing"
           : (flags & 2) ? "a column index is outside [0, n)"
                         : "the chains are not consecutive runs covering the rows";
}

}  // namespace cicy
