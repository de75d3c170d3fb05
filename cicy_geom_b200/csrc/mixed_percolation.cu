// Clusters and percolation of a mixed CNT/GNP network on the device
// (Determine_clusters_and_percolation for GNP_CNT_mix after Make_mixed_clusters,
// Hoshen_Kopelman.cpp:17-201, 2331-2903):
//   Make_particle_clusters  particles in window order grouped by label
//   Find_percolated_clusters a label percolates along x / y / z when a particle on face
//                           2 / 3 / 0 and one on face 4 / 5 / 1 carry it (CNT and GNP
//                           face lists alike); direction code 10 d + 1, family from the sum
//   Group_junctions         each junction to the percolated cluster of its particles' label
//   Remove_gnp_points_in_non_relevant_boundaries
//                           a GNP of a family 0-5 cluster drops its boundary points on faces
//                           the family does not use (unless they are junction points)
// One pass of kernels per step; the lists come back to the host in upstream's order
// (label order, window order inside a label, junction order inside a group).
#include <algorithm>
#include <string>
#include <vector>

#include "ctx.cuh"

namespace cicy {

namespace {

int grid_of(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    return (int)std::max(1LL, std::min(b, 148LL * 32));
}

// face bits per label: particles of the six face lists (CNT entries first, then GNP entries)
__global__ void k_label_faces(int n, const int32_t* __restrict__ part, const int32_t* __restrict__ face, const int32_t* __restrict__ is_gnp,
                              const int32_t* __restrict__ labels_cnt, const int32_t* __restrict__ labels_gnp, int32_t* __restrict__ bits) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int L = is_gnp[i] ? labels_gnp[part[i]] : labels_cnt[part[i]];
        if (L >= 0) atomicOr(&bits[L], 1 << face[i]);
    }
}

// Family_map (Hoshen_Kopelman.cpp:2591-2622) of the percolated directions' code sum.
__global__ void k_label_family(int nl, const int32_t* __restrict__ bits, int32_t* __restrict__ perc, int32_t* __restrict__ family) {
    for (int L = blockIdx.x * blockDim.x + threadIdx.x; L < nl; L += gridDim.x * blockDim.x) {
        const int b = bits[L];
        int sum = 0;
        const int pairs[3][2] = {{2, 4}, {3, 5}, {0, 1}};
        for (int d = 0; d < 3; d++)
            if ((b >> pairs[d][0] & 1) && (b >> pairs[d][1] & 1)) sum += 10 * d + 1;
        const int fam = sum == 1 ? 0 : sum == 11 ? 1 : sum == 21 ? 2 : sum == 12 ? 3 : sum == 22 ? 4 : sum == 32 ? 5 : sum == 33 ? 6 : -1;
        perc[L] = sum ? 1 : 0;
        family[L] = fam;
    }
}

// Sort keys of the particles inside: (label + 1, window position); label -1 first.
__global__ void k_member_keys(int n, const int32_t* __restrict__ inside, const int32_t* __restrict__ labels, uint64_t* __restrict__ key,
                              uint32_t* __restrict__ val) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = inside[i];
        key[i] = ((uint64_t)(uint32_t)(labels[p] + 1) << 32) | (uint32_t)i;
        val[i] = (uint32_t)p;
    }
}

// Group_junctions (Hoshen_Kopelman.cpp:2624-2710): junction k goes to the percolated cluster of
// its particles' label (key: cluster, k), or last when that label does not percolate.
__global__ void k_junction_keys(int n, const int32_t* __restrict__ n1, const int32_t* __restrict__ n2, const int32_t* __restrict__ l1,
                                const int32_t* __restrict__ l2, const int32_t* __restrict__ perc, const int32_t* __restrict__ perc_index,
                                int none, uint64_t* __restrict__ key, uint32_t* __restrict__ val, int* status) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int a = l1[n1[k]], b = l2[n2[k]];
        if (a != b) atomicCAS(status, 0, (int)DEV_INPUT);  // "junction particles have different labels"
        const int grp = (a >= 0 && perc[a]) ? perc_index[a] : none;
        key[k] = ((uint64_t)(uint32_t)grp << 32) | (uint32_t)k;
        val[k] = (uint32_t)k;
    }
}

// Check_relevant_boundary_and_remove_if_needed (Hoshen_Kopelman.cpp:2840-2880): per GNP of a
// percolated cluster of family 0-5, keep[e] says whether boundary entry e stays; a dropped
// entry's point leaves the GNP's list (marked in drop_pt).
__global__ void k_relevant_points(int ng, const int32_t* __restrict__ labels_gnp, const int32_t* __restrict__ perc,
                                  const int32_t* __restrict__ family, const int64_t* __restrict__ pb_ptr, const int64_t* __restrict__ pb_point,
                                  const int32_t* __restrict__ pb_face, const int32_t* __restrict__ bp, int32_t* __restrict__ keep,
                                  int32_t* __restrict__ drop_pt) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
        const int L = labels_gnp[g];
        const int fam = (L >= 0 && perc[L]) ? family[L] : 6;
        int r[4], nr = 0;
        switch (fam) {
            case 0: r[0] = 2; r[1] = 4; nr = 2; break;
            case 1: r[0] = 3; r[1] = 5; nr = 2; break;
            case 2: r[0] = 0; r[1] = 1; nr = 2; break;
            case 3: r[0] = 2; r[1] = 4; r[2] = 3; r[3] = 5; nr = 4; break;
            case 4: r[0] = 2; r[1] = 4; r[2] = 0; r[3] = 1; nr = 4; break;
            case 5: r[0] = 3; r[1] = 5; r[2] = 0; r[3] = 1; nr = 4; break;
            default: nr = 0;
        }
        for (int64_t e = pb_ptr[g]; e < pb_ptr[g + 1]; e++) {
            bool k = true;
            if (nr > 0) {
                const int f = pb_face[e];
                bool rel = false;
                for (int q = 0; q < nr; q++) rel |= (f == r[q]);
                k = rel || bp[pb_point[e]] != 0;
            }
            keep[e] = k ? 1 : 0;
            if (!k) drop_pt[pb_point[e]] = 1;
        }
    }
}

template <class T>
void up(Ctx& c, DBuf<T>& d, const T* h, size_t n) {
    d.ensure(std::max<size_t>(n, 1));
    if (n) CICY_CUDA(cudaMemcpyAsync(d.get(), h, sizeof(T) * n, cudaMemcpyHostToDevice, c.stream));
}

template <class T>
void down(Ctx& c, std::vector<T>& h, const DBuf<T>& d, size_t n) {
    h.resize(n);
    if (n) CICY_CUDA(cudaMemcpyAsync(h.data(), d.get(), sizeof(T) * n, cudaMemcpyDeviceToHost, c.stream));
}

// Sorted (key, val) pairs of n entries; key bits as given.
void sort_pairs(Ctx& c, DBuf<uint64_t>& k, DBuf<uint32_t>& v, int n, int bits) {
    if (n > 1) radix_sort_pairs(k.get(), v.get(), n, bits, c.rs, c.stream, c.launches);
}

}  // namespace

void run_mixed_percolation(Ctx& c, const cicy_mixed_state& in, MixedClusters& out) {
    auto bad = [](const std::string& m) { throw Fail{CICY_E_INPUT, "cicy_mixed_percolation: " + m}; };
    const int NL = in.n_labels, NC = in.n_cnts, NG = in.n_gnps;
    if (NL < 0 || NC < 0 || NG < 0 || in.n_cnts_inside < 0 || in.n_gnps_inside < 0 || in.n_points_gnp < 0) bad("negative sizes");
    for (int i = 0; i < NC; i++)
        if (in.labels_cnt[i] < -1 || in.labels_cnt[i] >= NL) bad("CNT label out of range");
    for (int i = 0; i < NG; i++)
        if (in.labels_gnp[i] < -1 || in.labels_gnp[i] >= NL) bad("GNP label out of range");
    for (int i = 0; i < in.n_cnts_inside; i++)
        if (in.cnts_inside[i] < 0 || in.cnts_inside[i] >= NC) bad("cnts_inside out of range");
    for (int i = 0; i < in.n_gnps_inside; i++)
        if (in.gnps_inside[i] < 0 || in.gnps_inside[i] >= NG) bad("gnps_inside out of range");
    // face entries: CNTs of the six faces, then GNPs
    std::vector<int32_t> fpart, fface, fgnp;
    for (int f = 0; f < 6; f++) {
        for (int64_t k = in.boundary_cnt_ptr[f]; k < in.boundary_cnt_ptr[f + 1]; k++) {
            if (in.boundary_cnt_idx[k] < 0 || in.boundary_cnt_idx[k] >= NC) bad("boundary_cnt out of range");
            fpart.push_back(in.boundary_cnt_idx[k]); fface.push_back(f); fgnp.push_back(0);
        }
        for (int64_t k = in.boundary_gnp_ptr[f]; k < in.boundary_gnp_ptr[f + 1]; k++) {
            if (in.boundary_gnp_idx[k] < 0 || in.boundary_gnp_idx[k] >= NG) bad("boundary_gnp out of range");
            fpart.push_back(in.boundary_gnp_idx[k]); fface.push_back(f); fgnp.push_back(1);
        }
    }
    auto chk_pairs = [&](int64_t n, const int32_t* a, int na, const int32_t* b, int nb2, const char* what) {
        for (int64_t k = 0; k < n; k++)
            if (a[k] < 0 || a[k] >= na || b[k] < 0 || b[k] >= nb2) bad(std::string(what) + " out of range");
    };
    chk_pairs(in.n_junctions_cnt, in.jc_n1, NC, in.jc_n2, NC, "CNT junction");
    chk_pairs(in.n_junctions_gnp, in.jg_n1, NG, in.jg_n2, NG, "GNP junction");
    chk_pairs(in.n_junctions_mixed, in.jm_n1, NC, in.jm_n2, NG, "mixed junction");
    if (NG > 0 && (!in.structure_gnp_ptr || !in.pts_boundary_ptr || !in.bp_flags)) bad("GNP lists missing");
    for (int g = 0; g < NG; g++) {
        for (int64_t k = in.structure_gnp_ptr[g]; k < in.structure_gnp_ptr[g + 1]; k++)
            if (in.structure_gnp_idx[k] < 0 || in.structure_gnp_idx[k] >= in.n_points_gnp) bad("structure_gnp out of range");
        for (int64_t k = in.pts_boundary_ptr[g]; k < in.pts_boundary_ptr[g + 1]; k++)
            if (in.pts_boundary_point[k] < 0 || in.pts_boundary_point[k] >= in.n_points_gnp || in.pts_boundary_face[k] < 0 ||
                in.pts_boundary_face[k] > 5)
                bad("pts_boundary out of range");
    }
    cudaStream_t s = c.stream;
    DBuf<int32_t> lc, lg, part, face, isg, bits, perc, fam, pidx, inside, n1, n2, keep, drop, bp, pbf, tmp;
    DBuf<int64_t> pbp, pbpt;
    DBuf<uint64_t> key;
    DBuf<uint32_t> val;
    up(c, lc, in.labels_cnt, NC);
    up(c, lg, in.labels_gnp, NG);
    const int NF = (int)fpart.size();
    up(c, part, fpart.data(), NF);
    up(c, face, fface.data(), NF);
    up(c, isg, fgnp.data(), NF);
    bits.ensure(std::max(NL, 1));
    perc.ensure(std::max(NL, 1));
    fam.ensure(std::max(NL, 1));
    pidx.ensure(std::max(NL, 1) + 1);
    CICY_CUDA(cudaMemsetAsync(bits.get(), 0, sizeof(int32_t) * std::max(NL, 1), s));
    if (NF) k_label_faces<<<grid_of(NF), 256, 0, s>>>(NF, part.get(), face.get(), isg.get(), lc.get(), lg.get(), bits.get());
    k_label_family<<<grid_of(NL), 256, 0, s>>>(NL, bits.get(), perc.get(), fam.get());
    exclusive_scan_i32(perc.get(), pidx.get(), NL, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
    c.launches += 2;
    const int NP = read_i32(c, c.i32_scalar.get());
    std::vector<int32_t> hperc, hfam;
    down(c, hperc, perc, NL);
    down(c, hfam, fam, NL);
    // Make_particle_clusters: members in window order, grouped by label (label -1 first)
    auto members = [&](const int32_t* ins, int n, DBuf<int32_t>& labels, std::vector<int64_t>& cptr, std::vector<int32_t>& cidx,
                       std::vector<int64_t>& iptr, std::vector<int32_t>& iidx) {
        up(c, inside, ins, n);
        key.ensure(std::max(n, 1));
        val.ensure(std::max(n, 1));
        if (n) k_member_keys<<<grid_of(n), 256, 0, s>>>(n, inside.get(), labels.get(), key.get(), val.get());
        sort_pairs(c, key, val, n, 32 + bits_for((uint64_t)NL + 1));
        std::vector<uint64_t> hk;
        std::vector<uint32_t> hv;
        down(c, hk, key, n);
        down(c, hv, val, n);
        CICY_CUDA(cudaStreamSynchronize(s));
        // per label the run of its members; percolated labels in label order are the clusters,
        // label -1 and the other labels in label order the isolated lists
        std::vector<int64_t> start(NL + 2, 0);
        for (int i = 0; i < n; i++) start[(hk[i] >> 32) + 1]++;
        for (int L = 0; L <= NL; L++) start[L + 1] += start[L];
        cptr.assign(1, 0);
        iptr.assign(1, 0);
        cidx.clear();
        iidx.clear();
        auto take = [&](int grp, std::vector<int64_t>& ptr, std::vector<int32_t>& idx) {
            for (int64_t i = start[grp]; i < start[grp + 1]; i++) idx.push_back((int32_t)hv[i]);
            ptr.push_back((int64_t)idx.size());
        };
        take(0, iptr, iidx);
        for (int L = 0; L < NL; L++) {
            if (hperc[L]) take(L + 1, cptr, cidx);
            else take(L + 1, iptr, iidx);
        }
    };
    members(in.cnts_inside, in.n_cnts_inside, lc, out.clu_cnt_ptr, out.clu_cnt, out.iso_cnt_ptr, out.iso_cnt);
    members(in.gnps_inside, in.n_gnps_inside, lg, out.clu_gnp_ptr, out.clu_gnp, out.iso_gnp_ptr, out.iso_gnp);
    out.family.clear();
    for (int L = 0; L < NL; L++)
        if (hperc[L]) out.family.push_back(hfam[L]);
    // Group_junctions
    auto group = [&](int64_t n, const int32_t* a, const int32_t* b, DBuf<int32_t>& la, DBuf<int32_t>& lb, std::vector<int64_t>& ptr,
                     std::vector<int32_t>& idx) {
        const int N = (int)n;
        up(c, n1, a, N);
        up(c, n2, b, N);
        key.ensure(std::max(N, 1));
        val.ensure(std::max(N, 1));
        if (N) k_junction_keys<<<grid_of(N), 256, 0, s>>>(N, n1.get(), n2.get(), la.get(), lb.get(), perc.get(), pidx.get(), NP, key.get(), val.get(),
                                                         c.status.get());
        sort_pairs(c, key, val, N, 32 + bits_for((uint64_t)NP + 1));
        std::vector<uint64_t> hk;
        std::vector<uint32_t> hv;
        down(c, hk, key, N);
        down(c, hv, val, N);
        check_status(c, "Group_junctions (junction particles with different labels)");
        ptr.assign(NP + 1, 0);
        idx.clear();
        for (int i = 0; i < N; i++) {
            const int grp = (int)(hk[i] >> 32);
            if (grp >= NP) break;
            idx.push_back((int32_t)hv[i]);
            ptr[grp + 1]++;
        }
        for (int q = 0; q < NP; q++) ptr[q + 1] += ptr[q];
    };
    group(in.n_junctions_cnt, in.jc_n1, in.jc_n2, lc, lc, out.jc_ptr, out.jc);
    group(in.n_junctions_gnp, in.jg_n1, in.jg_n2, lg, lg, out.jg_ptr, out.jg);
    group(in.n_junctions_mixed, in.jm_n1, in.jm_n2, lc, lg, out.jm_ptr, out.jm);
    // Remove_gnp_points_in_non_relevant_boundaries (only when something percolates)
    const int64_t NE = NG ? in.pts_boundary_ptr[NG] : 0;
    out.st_ptr.assign(NG + 1, 0);
    out.pb_ptr.assign(NG + 1, 0);
    out.st_idx.clear();
    out.pb_point.clear();
    out.pb_face.clear();
    std::vector<int32_t> hkeep((size_t)NE, 1), hdrop;
    if (NP > 0 && NE > 0) {
        up(c, pbp, in.pts_boundary_ptr, (size_t)NG + 1);
        up(c, pbpt, in.pts_boundary_point, (size_t)NE);
        up(c, pbf, in.pts_boundary_face, (size_t)NE);
        up(c, bp, in.bp_flags, (size_t)in.n_points_gnp);
        keep.ensure((size_t)NE);
        drop.ensure(std::max<int64_t>(in.n_points_gnp, 1));
        CICY_CUDA(cudaMemsetAsync(drop.get(), 0, sizeof(int32_t) * std::max<int64_t>(in.n_points_gnp, 1), s));
        k_relevant_points<<<grid_of(NG), 256, 0, s>>>(NG, lg.get(), perc.get(), fam.get(), pbp.get(), pbpt.get(), pbf.get(), bp.get(), keep.get(),
                                                      drop.get());
        c.launches++;
        down(c, hkeep, keep, (size_t)NE);
        down(c, hdrop, drop, (size_t)in.n_points_gnp);
    }
    CICY_LAUNCH_CHECK();
    CICY_CUDA(cudaStreamSynchronize(s));
    for (int g = 0; g < NG; g++) {
        for (int64_t k = in.structure_gnp_ptr[g]; k < in.structure_gnp_ptr[g + 1]; k++) {
            const int64_t P = in.structure_gnp_idx[k];
            if (hdrop.empty() || !hdrop[P]) out.st_idx.push_back(P);
        }
        out.st_ptr[g + 1] = (int64_t)out.st_idx.size();
        for (int64_t e = in.pts_boundary_ptr[g]; e < in.pts_boundary_ptr[g + 1]; e++)
            if (hkeep[e]) {
                out.pb_point.push_back(in.pts_boundary_point[e]);
                out.pb_face.push_back(in.pts_boundary_face[e]);
            }
        out.pb_ptr[g + 1] = (int64_t)out.pb_point.size();
    }
}

}  // namespace cicy
