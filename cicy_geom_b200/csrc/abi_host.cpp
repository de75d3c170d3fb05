// C ABI entry points for the host-side network sources (cicy_b200.h).
#include <new>

#include "cicy_internal.h"

namespace {
thread_local std::string g_host_error;
}

namespace cicy {
void set_host_error(const std::string& msg) { g_host_error = msg; }
}  // namespace cicy

extern "C" {

cicy_status cicy_generate_cnt_network(const cicy_gen_params* g, cicy_host_network** out) {
    if (!g || !out || g->n_cnts < 0 || g->step <= 0 || g->len_max < g->len_min || g->len_min < 0 || g->radius < 0)
        return CICY_E_INPUT;
    cicy::HostNetwork* h = cicy::generate_cnt_network(*g);
    cicy_host_network* w = new (std::nothrow) cicy_host_network;
    if (!w) { delete h; return CICY_E_INTERNAL; }
    w->net = std::move(*h);
    delete h;
    *out = w;
    return CICY_OK;
}

cicy_status cicy_extract_window(const cicy_host_network* in, const cicy_window_params* p, cicy_host_network** out) {
    if (!in || !p || !out) return CICY_E_INPUT;
    cicy::HostNetwork* h = nullptr;
    cicy_status s = cicy::extract_window(in->net, *p, &h, g_host_error);
    if (s != CICY_OK) return s;
    cicy_host_network* w = new cicy_host_network;
    w->net = std::move(*h);
    delete h;
    *out = w;
    return CICY_OK;
}

cicy_status cicy_read_network(const char* directory, int32_t file_type, cicy_host_network** out) {
    if (!directory || !out) return CICY_E_INPUT;
    cicy::HostNetwork* h = nullptr;
    cicy_status s = cicy::read_network_files(directory, file_type, &h, g_host_error);
    if (s != CICY_OK) return s;
    cicy_host_network* w = new cicy_host_network;
    w->net = std::move(*h);
    delete h;
    *out = w;
    return CICY_OK;
}

cicy_status cicy_read_gnps(const char* directory, cicy_gnp_set** out) {
    if (!directory || !out) return CICY_E_INPUT;
    cicy::GnpSet* g = nullptr;
    cicy_status s = cicy::read_gnp_file(directory, &g, g_host_error);
    if (s != CICY_OK) return s;
    cicy_gnp_set* w = new cicy_gnp_set;
    w->g = std::move(*g);
    delete g;
    *out = w;
    return CICY_OK;
}

cicy_status cicy_gnp_set_view(const cicy_gnp_set* set, cicy_gnps* view) {
    if (!set || !view) return CICY_E_INPUT;
    const cicy::GnpSet& g = set->g;
    view->n = g.n;
    view->l = g.l.data();
    view->t = g.t.data();
    view->center = g.center.data();
    view->rotation = g.rotation.data();
    view->vertices = g.vertices.data();
    view->planes = g.planes.data();
    return CICY_OK;
}

void cicy_gnp_set_free(cicy_gnp_set* set) { delete set; }

cicy_status cicy_host_network_from_arrays(const cicy_network* n, cicy_host_network** out) {
    if (!n || !out || n->n_points < 0 || n->n_cnts < 0 || !n->structure_ptr) return CICY_E_INPUT;
    cicy::HostNetwork* h = cicy::host_network_from_view(*n);
    cicy_host_network* w = new cicy_host_network;
    w->net = std::move(*h);
    delete h;
    *out = w;
    return CICY_OK;
}

cicy_status cicy_host_network_view(const cicy_host_network* h, cicy_network* v) {
    if (!h || !v) return CICY_E_INPUT;
    cicy::host_network_view(h->net, *v);
    return CICY_OK;
}

void cicy_host_network_free(cicy_host_network* h) { delete h; }

const char* cicy_host_last_error(void) { return g_host_error.c_str(); }


cicy_status cicy_gnp_extract_window(const cicy_gnp_set* gnps, const cicy_window_params* w, cicy_gnp_window** out) {
    if (!gnps || !w || !out) {
        cicy::set_host_error("cicy_gnp_extract_window: null argument");
        return CICY_E_INPUT;
    }
    *out = nullptr;
    cicy_gnp_window* h = new cicy_gnp_window;
    std::string err;
    const cicy_status st = cicy::gnp_window(gnps->g, *w, h->w, err);
    if (st != CICY_OK) {
        cicy::set_host_error(err);
        delete h;
        return st;
    }
    auto flat = [](const std::vector<std::vector<int32_t>>& v, std::vector<int32_t>& ptr, std::vector<int32_t>& idx) {
        ptr.assign(1, 0);
        idx.clear();
        for (const auto& r : v) {
            idx.insert(idx.end(), r.begin(), r.end());
            ptr.push_back((int32_t)idx.size());
        }
    };
    cicy::GnpWindow& g = h->w;
    flat(g.boundary_gnp, g.flat_bgnp_ptr, g.flat_bgnp_idx);
    flat(g.boundary_pts, g.flat_bpts_ptr, g.flat_bpts_idx);
    flat(g.structure, g.flat_st_ptr, g.flat_st_idx);
    *out = h;
    return CICY_OK;
}

cicy_status cicy_gnp_window_view(const cicy_gnp_window* h, cicy_gnp_window_list* v) {
    if (!h || !v) return CICY_E_INPUT;
    const cicy::GnpWindow& g = h->w;
    v->n_inside = (int32_t)g.inside.size();
    v->gnps_inside = g.inside.data();
    v->boundary_gnp_ptr = g.flat_bgnp_ptr.data();
    v->boundary_gnp_idx = g.flat_bgnp_idx.data();
    v->n_points = (int64_t)g.point_gnp.size();
    v->points = g.points.data();
    v->point_gnp = g.point_gnp.data();
    v->point_boundary = g.point_boundary.data();
    v->boundary_pts_ptr = g.flat_bpts_ptr.data();
    v->boundary_pts_idx = g.flat_bpts_idx.data();
    v->n_gnps = (int32_t)g.structure.size();
    v->structure_ptr = g.flat_st_ptr.data();
    v->structure_idx = g.flat_st_idx.data();
    v->volume = g.volume.data();
    return CICY_OK;
}

void cicy_gnp_window_free(cicy_gnp_window* h) { delete h; }
}  // extern "C"
