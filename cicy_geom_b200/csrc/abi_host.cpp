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

}  // extern "C"
