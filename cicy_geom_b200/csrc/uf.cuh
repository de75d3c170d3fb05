// Lock-free union-find on the device: hook the larger root under the smaller
// one (so parent[x] <= x always, and every walk ends), path halving while
// uniting.  Loads of parent[] bypass L1 (__ldcg): another SM's CAS must be
// visible to the retry loop.
#pragma once

#include <cstdint>

namespace cicy {

__device__ __forceinline__ int uf_find(int32_t* parent, int x) {
    while (true) {
        int p = __ldcg(&parent[x]);
        if (p == x) return x;
        int gp = __ldcg(&parent[p]);
        if (gp != p) parent[x] = gp;
        x = p;
    }
}

// Read-only find for the flattening pass: a writing find there could store a
// stale, non-root ancestor over a parent[] entry another thread already finalised.
__device__ __forceinline__ int uf_root(const int32_t* parent, int x) {
    while (true) {
        int p = __ldcg(&parent[x]);
        if (p == x) return x;
        x = p;
    }
}

__device__ __forceinline__ void uf_unite(int32_t* parent, int a, int b) {
    while (true) {
        int ra = uf_find(parent, a), rb = uf_find(parent, b);
        if (ra == rb) return;
        if (ra > rb) {
            const int t = ra;
            ra = rb;
            rb = t;
        }
        if (atomicCAS(&parent[rb], rb, ra) == rb) return;
    }
}

}  // namespace cicy
