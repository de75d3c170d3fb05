// Host build of the device geometry headers (test helper): the same source the
// CUDA kernels compile, built by g++ without FMA contraction, run on arrays
// from a file so the CPU tests can compare it with the upstream fixtures.
//
//   host_geometry <mode> <in.bin> <out.bin>
//
// in.bin: int32 n_gnps, n_items; double V[24 n_gnps], F[24 n_gnps]; then per mode
//   closest:  double q[4 n_items] (x, y, z, GNP)       -> double (flag, dist, qx, qy, qz) per item
//   pairs:    double p[2 n_items] (a, b); double vdw   -> double (status, penetrating, dist, N3, disp3)
//   junction: double p[2 n_items]; double vdw, lo[3], hi[3]
//                                                      -> double (distance status, junction status, outside, PA3, PB3)
//   triangulate (own layout): int32 n_gnps, n_points; double points[3 n_points];
//             int32 ptr[n_gnps + 1], idx[ptr[n_gnps]]; double l[n_gnps], centre[3 n_gnps],
//             rotation[9 n_gnps], planes[24 n_gnps]  -> int32 edge_ptr[n_gnps + 1], edges[2 E]
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#define __host__
#define __device__
#include "gnp_gjk.cuh"
#include "gnp_junction.cuh"
#include "gnp_triangulation.cuh"

using namespace cicy::gnp;

template <class T>
bool get(FILE* f, std::vector<T>& v, size_t n) {
    v.resize(n);
    return fread(v.data(), sizeof(T), n, f) == n;
}

int triangulate_all(FILE* f, const char* out_path) {
    int hdr[2];
    if (fread(hdr, 4, 2, f) != 2) return 3;
    const int n_gnps = hdr[0], n_points = hdr[1];
    std::vector<double> pts, l, c, M, F;
    std::vector<int> ptr, idx;
    if (!get(f, pts, 3 * (size_t)n_points) || !get(f, ptr, n_gnps + 1) || !get(f, idx, ptr[n_gnps]) || !get(f, l, n_gnps) ||
        !get(f, c, 3 * (size_t)n_gnps) || !get(f, M, 9 * (size_t)n_gnps) || !get(f, F, 24 * (size_t)n_gnps))
        return 3;
    static TriWork<256> w;
    std::vector<int> eptr(1, 0), edges, buf(2 * 3 * TriWork<256>::kTris);
    for (int g = 0; g < n_gnps; g++) {
        const int k = triangulate<256>(pts.data(), idx.data() + ptr[g], ptr[g + 1] - ptr[g], l[g], &c[3 * (size_t)g], &M[9 * (size_t)g],
                                       normal(&F[24 * (size_t)g], 0), w, buf.data(), (int)buf.size() / 2);
        if (k < 0) return 5;
        edges.insert(edges.end(), buf.begin(), buf.begin() + 2 * k);
        eptr.push_back((int)edges.size() / 2);
    }
    FILE* o = fopen(out_path, "wb");
    if (!o) return 4;
    fwrite(eptr.data(), 4, eptr.size(), o);
    fwrite(edges.data(), 4, edges.size(), o);
    fclose(o);
    return 0;
}

int main(int argc, char** argv) {
    if (argc != 4) return 1;
    FILE* f = fopen(argv[2], "rb");
    if (!f) return 2;
    if (std::string(argv[1]) == "triangulate") return triangulate_all(f, argv[3]);
    int n_gnps = 0, n = 0;
    if (fread(&n_gnps, 4, 1, f) != 1 || fread(&n, 4, 1, f) != 1) return 3;
    std::vector<double> V(24 * (size_t)n_gnps), F(24 * (size_t)n_gnps);
    if (fread(V.data(), 8, V.size(), f) != V.size() || fread(F.data(), 8, F.size(), f) != F.size()) return 3;
    const std::string mode = argv[1];
    const size_t per = mode == "closest" ? 4 : 2;
    std::vector<double> in(per * (size_t)n);
    if (fread(in.data(), 8, in.size(), f) != in.size()) return 3;
    double extra[7] = {0, 0, 0, 0, 0, 0, 0};
    const size_t n_extra = mode == "pairs" ? 1 : (mode == "junction" ? 7 : 0);
    if (n_extra && fread(extra, 8, n_extra, f) != n_extra) return 3;
    fclose(f);
    std::vector<double> out;
    static Polytope T;
    for (int i = 0; i < n; i++) {
        if (mode == "closest") {
            const int g = (int)in[4 * i + 3];
            P3 q{0, 0, 0};
            double d = 0;
            const int fl = closest_point(&V[24 * (size_t)g], &F[24 * (size_t)g], P3{in[4 * i], in[4 * i + 1], in[4 * i + 2]}, q, d);
            out.insert(out.end(), {(double)fl, d, q.x, q.y, q.z});
            continue;
        }
        const int a = (int)in[2 * i], b = (int)in[2 * i + 1];
        double d = 0;
        P3 N{0, 0, 0}, m{0, 0, 0};
        bool pen = false;
        const int st = pair_distance(&V[24 * (size_t)a], &V[24 * (size_t)b], extra[0], T, d, N, m, pen);
        if (mode == "pairs") {
            out.insert(out.end(), {(double)st, pen ? 1.0 : 0.0, d, N.x, N.y, N.z, m.x, m.y, m.z});
            continue;
        }
        Cuboid8 A, B;
        load_cuboid(&V[24 * (size_t)a], &F[24 * (size_t)a], A);
        if (pen) moved_cuboid(&V[24 * (size_t)b], m, B);
        else load_cuboid(&V[24 * (size_t)b], &F[24 * (size_t)b], B);
        P3 PA{0, 0, 0}, PB{0, 0, 0};
        const int js = st == kGjkOk ? junction_points(A, B, N, d, false, PA, PB) : -1;
        if (js == kJuncOk && pen) PB = sub(PB, m);
        const double o = js == kJuncOk ? (outside_box(PA, extra + 1, extra + 4) ? 1 : 0) + (outside_box(PB, extra + 1, extra + 4) ? 2 : 0) : -1;
        out.insert(out.end(), {(double)st, (double)js, o, PA.x, PA.y, PA.z, PB.x, PB.y, PB.z});
    }
    f = fopen(argv[3], "wb");
    if (!f) return 4;
    fwrite(out.data(), 8, out.size(), f);
    fclose(f);
    return 0;
}
