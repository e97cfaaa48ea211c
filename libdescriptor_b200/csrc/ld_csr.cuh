// ld_csr.cuh -- a warp's CSR neighbour segment staged into shared memory by
// cp.async: the kernels that give each centre row to one warp copy the next
// row's list (4 bytes per lane and entry, one commit group) while the current
// row computes, and read it from shared memory when its turn comes.
#pragma once

#include "ld_internal.h"

namespace ldb {

struct RowMeta {
    int i, n;        // centre atom, list length
    long long off;   // first list entry
};

// the row's centre and list segment (row_list maps batch rows to list rows
// where the launch gives one)
__device__ __forceinline__ RowMeta row_meta(const RowArgs &a, int row) {
    const int lrow = a.row_list ? a.row_list[row] : row;
    RowMeta m;
    m.i = a.row_centre ? a.row_centre[row] : row;
    m.off = a.nbl_begin ? a.nbl_begin[lrow] : a.off[lrow];
    m.n = (int)(a.off[lrow + 1] - a.off[lrow]);
    return m;
}

// by all lanes of the warp: post the copies of entries 0 .. min(n, cap) - 1
__device__ __forceinline__ void csr_prefetch(const RowArgs &a, const RowMeta &m, int cap, int *dst) {
    const int lane = threadIdx.x & 31;
    const int n = m.n < cap ? m.n : cap;
    for (int jj = lane; jj < n; jj += 32) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst + jj);
        const size_t g = __cvta_generic_to_global(a.nbl + m.off + jj);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(g) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// the lane's copies have landed (the hardware waits for this thread's own
// groups only); the warp then agrees before anyone reads the segment
__device__ __forceinline__ void csr_wait() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();
}

}  // namespace ldb
