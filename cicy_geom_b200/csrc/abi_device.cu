// C ABI entry points of the device hot path (cicy_b200.h): context, stages, copy-out.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>

#include "cicy_internal.h"
#include "ctx.cuh"

struct cicy_ctx {
    cicy::Ctx c;
};

struct cicy_mixed_clusters {
    cicy::MixedClusters m;
};

namespace {

template <class F>
cicy_status guarded(cicy_ctx* ctx, F&& f) {
    if (!ctx) return CICY_E_INPUT;
    try {
        CICY_CUDA(cudaSetDevice(ctx->c.device));
        f(ctx->c);
        ctx->c.err.clear();
        return CICY_OK;
    } catch (const cicy::Fail& e) {
        ctx->c.err = e.msg;
        if (ctx->c.side) cudaStreamSynchronize(ctx->c.side);  // no side-stream work outlives a failed call
        return e.status;
    } catch (const std::bad_alloc&) {
        ctx->c.err = "host allocation failed";
        if (ctx->c.side) cudaStreamSynchronize(ctx->c.side);
        return CICY_E_INTERNAL;
    }
}

template <class T>
void d2h(cicy::Ctx& c, T* h, const T* d, size_t n) {
    if (n && h) CICY_CUDA(cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, c.stream));
}

void sync(cicy::Ctx& c) { CICY_CUDA(cudaStreamSynchronize(c.stream)); }

}  // namespace

extern "C" {

cicy_status cicy_ctx_create(cicy_ctx** out, int device) {
    if (!out) return CICY_E_INPUT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return CICY_E_DEVICE;
    if (device < 0 || device >= ndev) return CICY_E_INPUT;
    cicy_ctx* ctx = new (std::nothrow) cicy_ctx;
    if (!ctx) return CICY_E_INTERNAL;
    ctx->c.device = device;
    cicy_status s = guarded(ctx, [](cicy::Ctx& c) {
        CICY_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        c.own_stream = true;
        CICY_CUDA(cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking));
        CICY_CUDA(cudaEventCreateWithFlags(&c.ev_main, cudaEventDisableTiming));
        CICY_CUDA(cudaEventCreateWithFlags(&c.ev_side, cudaEventDisableTiming));
        cudaDeviceProp prop;
        CICY_CUDA(cudaGetDeviceProperties(&prop, c.device));
        c.num_sms = prop.multiProcessorCount;
        if (!prop.cooperativeLaunch) throw cicy::Fail{CICY_E_DEVICE, "device lacks cooperative launch"};
        c.status.ensure(1);
        CICY_CUDA(cudaMemsetAsync(c.status.get(), 0, sizeof(int), c.stream));
        c.i32_scalar.ensure(8);
        c.i64_scalar.ensure(8);
    });
    if (s != CICY_OK) {
        delete ctx;
        return s;
    }
    *out = ctx;
    return CICY_OK;
}

cicy_status cicy_ctx_destroy(cicy_ctx* ctx) {
    if (!ctx) return CICY_OK;
    cudaSetDevice(ctx->c.device);
    if (ctx->c.stream) cudaStreamSynchronize(ctx->c.stream);
    if (ctx->c.side) cudaStreamSynchronize(ctx->c.side);
    if (ctx->c.own_stream && ctx->c.stream) cudaStreamDestroy(ctx->c.stream);
    if (ctx->c.side) cudaStreamDestroy(ctx->c.side);
    if (ctx->c.ev_main) cudaEventDestroy(ctx->c.ev_main);
    if (ctx->c.ev_side) cudaEventDestroy(ctx->c.ev_side);
    delete ctx;  // frees every device buffer of the context
    return CICY_OK;
}

cicy_status cicy_ctx_set_stream(cicy_ctx* ctx, void* stream) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (c.stream) CICY_CUDA(cudaStreamSynchronize(c.stream));
        if (c.side) CICY_CUDA(cudaStreamSynchronize(c.side));
        if (c.own_stream && c.stream) CICY_CUDA(cudaStreamDestroy(c.stream));
        c.stream = (cudaStream_t)stream;
        c.own_stream = false;
    });
}

void* cicy_ctx_stream(cicy_ctx* ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

cicy_status cicy_ctx_set_solver(cicy_ctx* ctx, const cicy_solver_opts* o) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!o || o->precision < 0 || o->precision > 1 || o->preconditioner < 0 || o->preconditioner > 3 || o->max_iter_factor <= 0)
            throw cicy::Fail{CICY_E_INPUT, "cicy_ctx_set_solver: invalid options"};
        c.solver = *o;
    });
}

cicy_status cicy_ctx_set_spin_limit(cicy_ctx* ctx, int64_t polls) {
    return guarded(ctx, [&](cicy::Ctx& c) { c.sw.spin_limit = polls > 0 ? (long long)polls : cicy::kSpinLimit; });
}

const char* cicy_last_error(const cicy_ctx* ctx) { return ctx ? ctx->c.err.c_str() : "null context"; }

int64_t cicy_ctx_kernel_launches(const cicy_ctx* ctx) { return ctx ? ctx->c.launches : 0; }

cicy_status cicy_upload_network(cicy_ctx* ctx, const cicy_network* net) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!net) throw cicy::Fail{CICY_E_INPUT, "null network"};
        cicy::upload_network(c, *net);
    });
}

cicy_status cicy_ctx_generate_cnt_network(cicy_ctx* ctx, const cicy_gen_params* g) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!g) throw cicy::Fail{CICY_E_INPUT, "cicy_ctx_generate_cnt_network: null parameters"};
        cicy::generate_network_device(c, *g);
    });
}

cicy_status cicy_ctx_extract_window(cicy_ctx* ctx, const cicy_window_params* w) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!w) throw cicy::Fail{CICY_E_INPUT, "cicy_ctx_extract_window: null parameters"};
        cicy::extract_window_device(c, *w);
    });
}

cicy_status cicy_get_network(cicy_ctx* ctx, int64_t* n_points, int32_t* n_cnts, int32_t* n_inside, int64_t* n_bcnt, int64_t* n_bpts,
                             double* x, double* y, double* z, int32_t* flag, int32_t* cnt_start, int32_t* cnt_len, double* radii,
                             int32_t* cnts_inside, int64_t* bcnt_ptr, int32_t* bcnt_idx, int64_t* bpts_ptr, int32_t* bpts_idx,
                             cicy_cuboid* window) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (c.stage < 1) throw cicy::Fail{CICY_E_STATE, "cicy_get_network: no network on the device"};
        const bool faces = c.h_bcnt_ptr.size() == 7 && c.h_bpts_ptr.size() == 7;
        const int64_t nb = faces ? c.h_bcnt_ptr[6] : 0, np = faces ? c.h_bpts_ptr[6] : 0;
        if (n_points) *n_points = c.n_points;
        if (n_cnts) *n_cnts = c.n_cnts;
        if (n_inside) *n_inside = c.n_inside;
        if (n_bcnt) *n_bcnt = nb;
        if (n_bpts) *n_bpts = np;
        if (window) *window = c.window;
        d2h(c, x, c.x.get(), c.n_points);
        d2h(c, y, c.y.get(), c.n_points);
        d2h(c, z, c.z.get(), c.n_points);
        d2h(c, flag, c.flag.get(), c.n_points);
        d2h(c, cnt_start, c.cstart.get(), c.n_cnts);
        d2h(c, cnt_len, c.clen.get(), c.n_cnts);
        d2h(c, radii, c.radii.get(), c.n_cnts);
        d2h(c, cnts_inside, c.inside.get(), c.n_inside);
        d2h(c, bcnt_idx, c.bcnt_idx.get(), nb);
        d2h(c, bpts_idx, c.bpts_idx.get(), np);
        for (int f = 0; f < 7; f++) {
            if (bcnt_ptr) bcnt_ptr[f] = faces ? c.h_bcnt_ptr[f] : 0;
            if (bpts_ptr) bpts_ptr[f] = faces ? c.h_bpts_ptr[f] : 0;
        }
        sync(c);
    });
}

cicy_status cicy_contact_grid(cicy_ctx* ctx, const cicy_params* p) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!p) throw cicy::Fail{CICY_E_INPUT, "null params"};
        cicy::run_contact_grid(c, *p);
    });
}

cicy_status cicy_clusters(cicy_ctx* ctx, const cicy_params* p) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!p) throw cicy::Fail{CICY_E_INPUT, "null params"};
        cicy::run_clusters(c, *p);
    });
}

cicy_status cicy_electrical_analysis(cicy_ctx* ctx, const cicy_params* p, cicy_result* out) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!p) throw cicy::Fail{CICY_E_INPUT, "null params"};
        if (out) std::memset(out, 0, sizeof(*out));
        cicy::run_electrical(c, *p, out);
        if (out) {
            out->n_slots = c.n_slots;
            out->n_point_contacts = c.n_uc;
            out->n_labels = c.n_labels;
            out->n_junctions = c.n_junc;
        }
    });
}

cicy_status cicy_network_to_conductance(cicy_ctx* ctx, const cicy_params* p, cicy_result* out) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!p) throw cicy::Fail{CICY_E_INPUT, "null params"};
        cudaEvent_t ev[4];
        for (auto& e : ev) CICY_CUDA(cudaEventCreate(&e));
        CICY_CUDA(cudaEventRecord(ev[0], c.stream));
        cicy::run_contact_grid(c, *p);
        CICY_CUDA(cudaEventRecord(ev[1], c.stream));
        cicy::run_clusters(c, *p);
        CICY_CUDA(cudaEventRecord(ev[2], c.stream));
        if (out) std::memset(out, 0, sizeof(*out));
        cicy::run_electrical(c, *p, out);
        CICY_CUDA(cudaEventRecord(ev[3], c.stream));
        CICY_CUDA(cudaEventSynchronize(ev[3]));
        float ms[3];
        cudaEventElapsedTime(&ms[0], ev[0], ev[1]);
        cudaEventElapsedTime(&ms[1], ev[1], ev[2]);
        cudaEventElapsedTime(&ms[2], ev[0], ev[3]);
        for (auto& e : ev) cudaEventDestroy(e);
        if (out) {
            out->n_slots = c.n_slots;
            out->n_point_contacts = c.n_uc;
            out->n_labels = c.n_labels;
            out->n_junctions = c.n_junc;
            out->stage_seconds[0] = ms[0] * 1e-3;
            out->stage_seconds[1] = ms[1] * 1e-3;
            out->stage_seconds[5] = ms[2] * 1e-3;
        }
    });
}

cicy_status cicy_gnp_cnt_contacts(cicy_ctx* ctx, const cicy_gnp_set* gnps, const cicy_gnp_grid* grid, const cicy_params* p,
                                  int32_t inside_is_error, int64_t* n_contacts) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!gnps || !grid || !p) throw cicy::Fail{CICY_E_INPUT, "cicy_gnp_cnt_contacts: null argument"};
        const int n = cicy::run_gnp_cnt_contacts(c, gnps->g, grid->grid, *p, inside_is_error);
        if (n_contacts) *n_contacts = n;
    });
}

cicy_status cicy_mixed_labels(cicy_ctx* ctx, const int32_t* labels_gnp, int32_t n_gnps, int32_t n_total_labels, int32_t* labels_cnt,
                              int32_t* labels_gnp_out, int32_t* n_clusters) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (n_gnps < 0 || (n_gnps > 0 && !labels_gnp)) throw cicy::Fail{CICY_E_INPUT, "cicy_mixed_labels: null GNP labels"};
        const int n = cicy::run_mixed_labels(c, labels_gnp, n_gnps, n_total_labels, labels_cnt, labels_gnp_out);
        if (n_clusters) *n_clusters = n;
    });
}

cicy_status cicy_mixed_junctions(cicy_ctx* ctx, int64_t n_points_gnp, int32_t min_points, int64_t* n_junctions) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (n_points_gnp < 0 || n_points_gnp >= (1LL << 31)) throw cicy::Fail{CICY_E_INPUT, "cicy_mixed_junctions: invalid point count"};
        const int n = cicy::run_mixed_junctions(c, (int)n_points_gnp, min_points, c.h_mixj, c.h_mixj_dist, c.h_mixj_points);
        if (n_junctions) *n_junctions = n;
    });
}

cicy_status cicy_get_mixed_junctions(cicy_ctx* ctx, int64_t* n, int64_t* cnt_point, int32_t* cnt, int64_t* gnp_point, int32_t* gnp, double* dist,
                                     double* points) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        const size_t J = c.h_mixj_dist.size();
        if (n) *n = (int64_t)J;
        for (size_t j = 0; j < J; j++) {
            if (cnt_point) cnt_point[j] = c.h_mixj[4 * j];
            if (cnt) cnt[j] = c.h_mixj[4 * j + 1];
            if (gnp_point) gnp_point[j] = c.h_mixj[4 * j + 2];
            if (gnp) gnp[j] = c.h_mixj[4 * j + 3];
            if (dist) dist[j] = c.h_mixj_dist[j];
            if (points)
                for (int d = 0; d < 3; d++) points[3 * j + d] = c.h_mixj_points[3 * j + d];
        }
    });
}

cicy_status cicy_get_gnp_cnt_contacts(cicy_ctx* ctx, int64_t* n, int64_t* point, int32_t* gnp, double* dist, double* closest) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        const int U = c.n_mix;
        if (n) *n = U;
        if (point && U) {
            std::vector<int32_t> h(U);
            d2h(c, h.data(), c.mix_point.get(), U);
            sync(c);
            for (int i = 0; i < U; i++) point[i] = h[i];
        }
        d2h(c, gnp, c.mix_gnp.get(), U);
        d2h(c, dist, c.mix_dist.get(), U);
        d2h(c, closest, c.mix_closest.get(), 3 * (size_t)U);
        sync(c);
    });
}

cicy_status cicy_get_sectioned_domain(cicy_ctx* ctx, int64_t* n_regions, int64_t* n_slots, int64_t* ptr, int64_t* idx) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (c.stage < 2) throw cicy::Fail{CICY_E_STATE, "no contact grid"};
        const int R = (int)c.grid.total, S = c.n_slots;
        if (n_regions) *n_regions = R;
        if (n_slots) *n_slots = S;
        if (ptr) {
            std::vector<int32_t> h(R + 1);
            d2h(c, h.data(), c.region_ptr.get(), R + 1);
            sync(c);
            for (int i = 0; i <= R; i++) ptr[i] = h[i];
        }
        if (idx && S > 0) {
            std::vector<uint32_t> q(S);
            std::vector<int32_t> tp(c.n_trav);
            d2h(c, q.data(), c.slot_sorted.get(), S);
            d2h(c, tp.data(), c.trav_pt.get(), c.n_trav);
            sync(c);
            for (int i = 0; i < S; i++) idx[i] = tp[q[i]];
        }
    });
}

cicy_status cicy_get_point_contacts(cicy_ctx* ctx, int64_t* n, int64_t* pa, int32_t* cnt_b, int64_t* pb, double* dist) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (c.stage < 3) throw cicy::Fail{CICY_E_STATE, "no clusters"};
        const int N = c.n_uc;
        if (n) *n = N;
        if (!pa && !cnt_b && !pb && !dist) return;
        std::vector<int32_t> a(N), b(N), qa(N), qb(N);
        std::vector<double> d(N);
        d2h(c, b.data(), c.uc_b.get(), N);
        d2h(c, qa.data(), c.uc_pa.get(), N);
        d2h(c, qb.data(), c.uc_pb.get(), N);
        d2h(c, d.data(), c.uc_d.get(), N);
        sync(c);
        std::vector<int> order(N);
        for (int i = 0; i < N; i++) order[i] = i;
        std::sort(order.begin(), order.end(), [&](int u, int v) { return qa[u] != qa[v] ? qa[u] < qa[v] : b[u] < b[v]; });
        for (int i = 0; i < N; i++) {
            int o = order[i];
            if (pa) pa[i] = qa[o];
            if (cnt_b) cnt_b[i] = b[o];
            if (pb) pb[i] = qb[o];
            if (dist) dist[i] = d[o];
        }
    });
}

cicy_status cicy_get_labels(cicy_ctx* ctx, int32_t* n_cnts, int32_t* n_labels, int32_t* labels) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (c.stage < 3) throw cicy::Fail{CICY_E_STATE, "no clusters"};
        if (n_cnts) *n_cnts = c.n_cnts;
        if (n_labels) *n_labels = c.n_labels;
        d2h(c, labels, c.labels.get(), c.n_cnts);
        sync(c);
    });
}

cicy_status cicy_get_junctions(cicy_ctx* ctx, int64_t* n, int64_t* p1, int32_t* n1, int64_t* p2, int32_t* n2, double* dist) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (c.stage < 3) throw cicy::Fail{CICY_E_STATE, "no clusters"};
        const int N = c.n_junc;
        if (n) *n = N;
        std::vector<int32_t> a(N), b(N);
        if (p1) { d2h(c, a.data(), c.j_p1.get(), N); sync(c); for (int i = 0; i < N; i++) p1[i] = a[i]; }
        if (p2) { d2h(c, b.data(), c.j_p2.get(), N); sync(c); for (int i = 0; i < N; i++) p2[i] = b[i]; }
        d2h(c, n1, c.j_n1.get(), N);
        d2h(c, n2, c.j_n2.get(), N);
        d2h(c, dist, c.j_d.get(), N);
        sync(c);
    });
}

cicy_status cicy_mixed_percolation(cicy_ctx* ctx, const cicy_mixed_state* in, cicy_mixed_clusters** out) {
    if (!out) return CICY_E_INPUT;
    *out = nullptr;
    cicy_mixed_clusters* h = new (std::nothrow) cicy_mixed_clusters;
    if (!h) return CICY_E_INTERNAL;
    const cicy_status st = guarded(ctx, [&](cicy::Ctx& c) {
        if (!in) throw cicy::Fail{CICY_E_INPUT, "cicy_mixed_percolation: null argument"};
        cicy::run_mixed_percolation(c, *in, h->m);
    });
    if (st != CICY_OK) {
        delete h;
        return st;
    }
    *out = h;
    return CICY_OK;
}

cicy_status cicy_mixed_clusters_view(const cicy_mixed_clusters* h, cicy_mixed_clusters_list* v) {
    if (!h || !v) return CICY_E_INPUT;
    const cicy::MixedClusters& m = h->m;
    v->n_percolated = (int32_t)m.family.size();
    v->family = m.family.data();
    v->clusters_cnt_ptr = m.clu_cnt_ptr.data();
    v->clusters_cnt_idx = m.clu_cnt.data();
    v->clusters_gnp_ptr = m.clu_gnp_ptr.data();
    v->clusters_gnp_idx = m.clu_gnp.data();
    v->n_isolated_cnt = (int32_t)m.iso_cnt_ptr.size() - 1;
    v->isolated_cnt_ptr = m.iso_cnt_ptr.data();
    v->isolated_cnt_idx = m.iso_cnt.data();
    v->n_isolated_gnp = (int32_t)m.iso_gnp_ptr.size() - 1;
    v->isolated_gnp_ptr = m.iso_gnp_ptr.data();
    v->isolated_gnp_idx = m.iso_gnp.data();
    v->cnt_junctions_ptr = m.jc_ptr.data();
    v->cnt_junctions_idx = m.jc.data();
    v->gnp_junctions_ptr = m.jg_ptr.data();
    v->gnp_junctions_idx = m.jg.data();
    v->mix_junctions_ptr = m.jm_ptr.data();
    v->mix_junctions_idx = m.jm.data();
    v->structure_gnp_ptr = m.st_ptr.data();
    v->structure_gnp_idx = m.st_idx.data();
    v->pts_boundary_ptr = m.pb_ptr.data();
    v->pts_boundary_point = m.pb_point.data();
    v->pts_boundary_face = m.pb_face.data();
    return CICY_OK;
}

void cicy_mixed_clusters_free(cicy_mixed_clusters* h) { delete h; }

cicy_status cicy_hybrid_electrical(cicy_ctx* ctx, const cicy_hybrid_state* st, const cicy_params* p, double resistivity_gnp_surf,
                                   double resistivity_gnp_t, cicy_result* out) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!st || !p) throw cicy::Fail{CICY_E_INPUT, "cicy_hybrid_electrical: null argument"};
        cicy::run_hybrid_electrical(c, *st, *p, resistivity_gnp_surf, resistivity_gnp_t, out);
    });
}

cicy_status cicy_get_hybrid_structure(cicy_ctx* ctx, int64_t* n_idx, int64_t* ptr, int64_t* idx) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!c.have_hybrid || !c.hy) throw cicy::Fail{CICY_E_STATE, "no hybrid electrical stage yet"};
        cicy::HybridDev& H = *c.hy;
        const int NG = H.n_gnps;
        std::vector<int32_t> sp(NG + 1), sc(std::max(NG, 1));
        if (NG) {
            d2h(c, sp.data(), H.sptr.get(), NG + 1);
            d2h(c, sc.data(), H.scount.get(), NG);
        }
        sync(c);
        int64_t tot = 0;
        if (ptr) ptr[0] = 0;
        std::vector<int32_t> buf;
        for (int g = 0; g < NG; g++) {
            if (idx && sc[g]) {
                buf.resize(sc[g]);
                d2h(c, buf.data(), H.sidx.get() + sp[g], sc[g]);
                sync(c);
                for (int k = 0; k < sc[g]; k++) idx[tot + k] = buf[k];
            }
            tot += sc[g];
            if (ptr) ptr[g + 1] = tot;
        }
        if (n_idx) *n_idx = tot;
    });
}

cicy_status cicy_get_hybrid_volumes(cicy_ctx* ctx, double* volumes30) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!c.have_hybrid || !c.hy) throw cicy::Fail{CICY_E_STATE, "no hybrid electrical stage yet"};
        if (!volumes30) throw cicy::Fail{CICY_E_INPUT, "null buffer"};
        double a[31], g[15];
        d2h(c, a, c.vol_acc.get(), 31);
        d2h(c, g, c.hy->vol_acc.get(), 15);
        sync(c);
        std::copy(a, a + 8, volumes30);            // volumes_cnt
        std::copy(g, g + 8, volumes30 + 8);        // volumes_gnp
        std::copy(a + 8, a + 15, volumes30 + 16);  // dead_branches
        std::copy(g + 8, g + 15, volumes30 + 23);  // dead_gnps
    });
}

cicy_status cicy_get_hybrid_junctions(cicy_ctx* ctx, int32_t cluster, int64_t* n_gnp, int32_t* gnp, int64_t* n_mix, int32_t* mix) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!c.have_hybrid || !c.hy) throw cicy::Fail{CICY_E_STATE, "no hybrid electrical stage yet"};
        cicy::HybridDev& H = *c.hy;
        if (cluster < 0 || cluster >= H.n_clusters) throw cicy::Fail{CICY_E_INPUT, "no such cluster"};
        const int ng = H.cgj_len[cluster], nm = H.cmj_len[cluster];
        if (n_gnp) *n_gnp = ng;
        if (n_mix) *n_mix = nm;
        if (gnp && ng) d2h(c, gnp, H.cgj_idx.get() + H.h_cgj_ptr[cluster], ng);
        if (mix && nm) d2h(c, mix, H.cmj_idx.get() + H.h_cmj_ptr[cluster], nm);
        sync(c);
    });
}

cicy_status cicy_get_volumes(cicy_ctx* ctx, double* volumes_cnt, double* dead_branches, double* total_volumes, double* fractions) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!c.have_volumes) throw cicy::Fail{CICY_E_STATE, "no volumes yet (cicy_electrical_analysis with simulation_scope < 2)"};
        double acc[31];
        d2h(c, acc, c.vol_acc.get(), 31);
        sync(c);
        if (volumes_cnt) std::copy(acc, acc + 8, volumes_cnt);
        if (dead_branches) std::copy(acc + 8, acc + 15, dead_branches);
        if (total_volumes) std::copy(acc + 15, acc + 23, total_volumes);
        if (fractions) std::copy(acc + 23, acc + 31, fractions);
    });
}

cicy_status cicy_get_elements(cicy_ctx* ctx, int32_t which, int64_t* n_cnts, int64_t* n_idx, int64_t* ptr, int64_t* idx) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (c.stage < 3) throw cicy::Fail{CICY_E_STATE, "no clusters"};
        if (which == 1 && !c.have_backbone) throw cicy::Fail{CICY_E_STATE, "no backbone yet"};
        const int NC = c.n_cnts;
        std::vector<int32_t> lo(NC), hi(NC);
        int n_elem = 0;
        std::vector<int32_t> mscan(c.n_points + 1);
        d2h(c, mscan.data(), c.mark_scan.get(), c.n_points + 1);
        sync(c);
        n_elem = mscan[c.n_points];
        if (which == 1) {
            d2h(c, lo.data(), c.bb_lo.get(), NC);
            d2h(c, hi.data(), c.bb_hi.get(), NC);
            sync(c);
        } else {
            for (int i = 0; i < NC; i++) {
                int b = c.h_clen[i] ? mscan[c.h_cstart[i]] : 0, e = c.h_clen[i] ? mscan[c.h_cstart[i] + c.h_clen[i]] : 0;
                lo[i] = e > b ? b : -1;
                hi[i] = e > b ? e - 1 : -2;
            }
        }
        std::vector<int32_t> el(std::max(n_elem, 1));
        d2h(c, el.data(), c.elem_idx.get(), n_elem);
        sync(c);
        int64_t total = 0;
        if (ptr) ptr[0] = 0;
        for (int i = 0; i < NC; i++) {
            int64_t len = lo[i] >= 0 ? (hi[i] - lo[i] + 1) : 0;
            if (idx)
                for (int64_t k = 0; k < len; k++) idx[total + k] = el[lo[i] + k];
            total += len;
            if (ptr) ptr[i + 1] = total;
        }
        if (n_cnts) *n_cnts = NC;
        if (n_idx) *n_idx = total;
    });
}

cicy_status cicy_get_clusters(cicy_ctx* ctx, int32_t which, int32_t* n_clusters, int64_t* n_idx, int64_t* ptr, int32_t* idx,
                              int32_t* family, int64_t* n_junc_idx, int64_t* junc_ptr, int32_t* junc_idx) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (c.stage < 3) throw cicy::Fail{CICY_E_STATE, "no clusters"};
        if (which == 1 && !c.have_backbone) throw cicy::Fail{CICY_E_STATE, "no backbone yet"};
        const int K = c.n_perc;
        if (n_clusters) *n_clusters = K;
        if (family)
            for (int k = 0; k < K; k++) family[k] = c.h_family[k];
        const std::vector<int32_t>& cp = c.h_clu_ptr;  // storage offsets are those of the percolation stage
        const std::vector<int32_t>& jp = c.h_cj_ptr;
        int64_t tot = 0, jtot = 0;
        if (ptr) ptr[0] = 0;
        if (junc_ptr) junc_ptr[0] = 0;
        for (int k = 0; k < K; k++) {
            int len = which == 1 ? c.bb_clu_len[k] : cp[k + 1] - cp[k];
            int jlen = which == 1 ? c.bb_cj_len[k] : jp[k + 1] - jp[k];
            const int32_t* src = which == 1 ? c.bbclu_idx.get() : c.clu_idx.get();
            const int32_t* jsrc = which == 1 ? c.bbcj_idx.get() : c.cj_idx.get();
            if (idx && len) d2h(c, idx + tot, src + cp[k], len);
            if (junc_idx && jlen) d2h(c, junc_idx + jtot, jsrc + jp[k], jlen);
            tot += len;
            jtot += jlen;
            if (ptr) ptr[k + 1] = tot;
            if (junc_ptr) junc_ptr[k + 1] = jtot;
        }
        sync(c);
        if (n_idx) *n_idx = tot;
        if (n_junc_idx) *n_junc_idx = jtot;
    });
}

cicy_status cicy_get_system(cicy_ctx* ctx, int32_t solve, int64_t* nodes, int64_t* reserved, int64_t* nnz_lower, int64_t* row_ptr,
                            int64_t* col_ind, double* values, double* diag, double* b, double* x0, double* voltages) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (solve < 0 || solve >= (int)c.systems.size()) throw cicy::Fail{CICY_E_INPUT, "no such solve"};
        cicy::DeaSystem& s = *c.systems[solve];
        const int n = (int)(s.nodes - s.reserved), m = (int)s.nnz_lower;
        if (nodes) *nodes = s.nodes;
        if (reserved) *reserved = s.reserved;
        if (nnz_lower) *nnz_lower = m;
        std::vector<int32_t> rp(n + 1), ci(std::max(m, 1));
        if (row_ptr) {
            d2h(c, rp.data(), s.row_ptr.get(), n + 1);
            sync(c);
            for (int i = 0; i <= n; i++) row_ptr[i] = rp[i];
        }
        if (col_ind) {
            d2h(c, ci.data(), s.col.get(), m);
            sync(c);
            for (int i = 0; i < m; i++) col_ind[i] = ci[i];
        }
        d2h(c, values, s.val.get(), m);
        d2h(c, diag, s.diag.get(), n);
        d2h(c, b, s.b.get(), n);
        d2h(c, x0, s.x0.get(), n);
        d2h(c, voltages, s.volt.get(), s.nodes);
        sync(c);
    });
}

cicy_status cicy_get_chains(cicy_ctx* ctx, int32_t solve, int32_t* n_chains, int32_t* start, int32_t* len) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (solve < 0 || solve >= (int)c.systems.size()) throw cicy::Fail{CICY_E_INPUT, "no such solve"};
        const cicy::DeaSystem& s = *c.systems[solve];
        const int m = (int)s.h_chain_start.size();
        if (n_chains) *n_chains = m;
        if (start) std::memcpy(start, s.h_chain_start.data(), sizeof(int32_t) * m);
        if (len) std::memcpy(len, s.h_chain_len.data(), sizeof(int32_t) * m);
    });
}

cicy_status cicy_ctx_set_learned_params(cicy_ctx* ctx, const float* params, int32_t n) {
    return guarded(ctx, [&](cicy::Ctx& c) {
        if (!params || n != cicy::gnn_param_count())
            throw cicy::Fail{CICY_E_INPUT, "cicy_ctx_set_learned_params: expected " + std::to_string(cicy::gnn_param_count()) + " parameters"};
        c.gnn_params.ensure(n);
        CICY_CUDA(cudaMemcpyAsync(c.gnn_params.get(), params, sizeof(float) * n, cudaMemcpyHostToDevice, c.stream));
        CICY_CUDA(cudaStreamSynchronize(c.stream));
    });
}

}  // extern "C"
