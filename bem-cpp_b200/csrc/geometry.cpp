// Host-side geometry: meshes, RWG basis, triangle quadrature, orientation
// quadrature.  Same results as the reference's mesh.cpp, rwg.cpp,
// quadrature.h and orient.cpp (cited per function); the RWG order is the
// reference C++ order (edges sorted by (min vertex, max vertex)).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <utility>

#include "bem_internal.h"

namespace bem {

static inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline double norm(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

double tri_area(const HostMesh& m, int t) {
    V3 v0 = m.verts[m.tris[3 * t]], v1 = m.verts[m.tris[3 * t + 1]], v2 = m.verts[m.tris[3 * t + 2]];
    return 0.5 * norm(cross(sub(v1, v0), sub(v2, v0)));
}

// One 1->4 midpoint split.  Edge midpoints are numbered in first-visit order;
// children (a,ab,ca), (b,bc,ab), (c,ca,bc), (ab,bc,ca) (mesh.cpp:27-56, :70-100).
static HostMesh split4(const HostMesh& in, bool project) {
    HostMesh out;
    out.verts = in.verts;
    std::map<std::pair<int, int>, int> mid;
    auto get_mid = [&](int a, int b) {
        std::pair<int, int> key(std::min(a, b), std::max(a, b));
        auto it = mid.find(key);
        if (it != mid.end()) return it->second;
        V3 p = scale(add(out.verts[a], out.verts[b]), 0.5);
        if (project) {
            double n = norm(p);
            p = {p.x / n, p.y / n, p.z / n};
        }
        int idx = (int)out.verts.size();
        out.verts.push_back(p);
        mid[key] = idx;
        return idx;
    };
    out.tris.reserve(in.tris.size() * 4);
    for (int t = 0; t < in.nt(); t++) {
        int a = in.tris[3 * t], b = in.tris[3 * t + 1], c = in.tris[3 * t + 2];
        int ab = get_mid(a, b), bc = get_mid(b, c), ca = get_mid(c, a);
        int ch[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
        out.tris.insert(out.tris.end(), ch, ch + 12);
    }
    return out;
}

// icosphere -- mesh.cpp:11-68
HostMesh make_icosphere(double radius, int refinements) {
    const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
    HostMesh m;
    m.verts = {{-1, phi, 0}, {1, phi, 0}, {-1, -phi, 0}, {1, -phi, 0},
               {0, -1, phi}, {0, 1, phi}, {0, -1, -phi}, {0, 1, -phi},
               {phi, 0, -1}, {phi, 0, 1}, {-phi, 0, -1}, {-phi, 0, 1}};
    double inv = 1.0 / norm(m.verts[0]);
    for (auto& v : m.verts) v = scale(v, inv);
    m.tris = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4,
              11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8,
              3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    for (int r = 0; r < refinements; r++) m = split4(m, true);
    for (auto& v : m.verts) v = scale(v, radius);
    return m;
}

HostMesh subdivide_flat(const HostMesh& m) { return split4(m, false); }

// hex_prism -- mesh.cpp:102-154: unit equivalent-sphere radius,
// a = (8 pi / (27 AR))^(1/3), H = AR a sqrt(3).
HostMesh make_hex_prism(double ar, int refinements) {
    double a = std::pow(8.0 * M_PI / (27.0 * ar), 1.0 / 3.0);
    double H = ar * a * std::sqrt(3.0);
    HostMesh m;
    m.verts.resize(14);
    m.verts[0] = {0, 0, H / 2};
    m.verts[7] = {0, 0, -H / 2};
    for (int i = 0; i < 6; i++) {
        double ang = 2.0 * M_PI * i / 6.0;
        double x = a * std::cos(ang), y = a * std::sin(ang);
        m.verts[1 + i] = {x, y, H / 2};
        m.verts[8 + i] = {x, y, -H / 2};
    }
    for (int i = 0; i < 6; i++) {
        int i1 = 1 + i, i2 = 1 + (i + 1) % 6, j1 = 8 + i, j2 = 8 + (i + 1) % 6;
        int t[12] = {0, i1, i2, 7, j2, j1, i1, j1, j2, i1, j2, i2};
        m.tris.insert(m.tris.end(), t, t + 12);
    }
    for (int r = 0; r < refinements; r++) m = split4(m, false);
    return m;
}

// build_rwg -- rwg.cpp:5-43.  Interior edges (shared by exactly two
// triangles) in (min,max) key order; the first visiting triangle is '+'.
HostRWG build_rwg(const HostMesh& m) {
    std::map<std::pair<int, int>, std::vector<std::pair<int, int>>> edges;
    for (int t = 0; t < m.nt(); t++)
        for (int j = 0; j < 3; j++) {
            int a = m.tris[3 * t + j], b = m.tris[3 * t + (j + 1) % 3];
            int opp = m.tris[3 * t + (j + 2) % 3];
            edges[{std::min(a, b), std::max(a, b)}].push_back({t, opp});
        }
    HostRWG r;
    for (auto& kv : edges) {
        if (kv.second.size() != 2) continue;
        int tp = kv.second[0].first, vp = kv.second[0].second;
        int tm = kv.second[1].first, vm = kv.second[1].second;
        r.tri_p.push_back(tp);
        r.tri_m.push_back(tm);
        r.vfree_p.push_back(vp);
        r.vfree_m.push_back(vm);
        r.free_p.push_back(m.verts[vp]);
        r.free_m.push_back(m.verts[vm]);
        r.length.push_back(norm(sub(m.verts[kv.first.second], m.verts[kv.first.first])));
        r.area_p.push_back(tri_area(m, tp));
        r.area_m.push_back(tri_area(m, tm));
        r.edge_lo.push_back(kv.first.first);
        r.edge_hi.push_back(kv.first.second);
    }
    r.N = (int)r.tri_p.size();
    return r;
}

void rwg_refresh(const HostMesh& m, HostRWG& r) {
    for (int n = 0; n < r.N; n++) {
        r.free_p[n] = m.verts[r.vfree_p[n]];
        r.free_m[n] = m.verts[r.vfree_m[n]];
        r.length[n] = norm(sub(m.verts[r.edge_hi[n]], m.verts[r.edge_lo[n]]));
        r.area_p[n] = tri_area(m, r.tri_p[n]);
        r.area_m[n] = tri_area(m, r.tri_m[n]);
    }
}

// Dunavant rules -- quadrature.h:14-70.  Barycentric (l1, l2), weights sum to 1.
bool quadrature(int order, Quad* q) {
    if (order == 4) {
        const double l1[4] = {1.0 / 3, 0.6, 0.2, 0.2}, l2[4] = {1.0 / 3, 0.2, 0.6, 0.2};
        const double w[4] = {-27.0 / 48, 25.0 / 48, 25.0 / 48, 25.0 / 48};
        q->n = 4;
        for (int i = 0; i < 4; i++) q->l1[i] = l1[i], q->l2[i] = l2[i], q->w[i] = w[i];
        return true;
    }
    if (order == 7) {
        const double a1 = 0.059715871789770, a2 = 0.470142064105115;
        const double b1 = 0.797426985353087, b2 = 0.101286507323456;
        const double l1[7] = {1.0 / 3, a1, a2, a2, b1, b2, b2};
        const double l2[7] = {1.0 / 3, a2, a1, a2, b2, b1, b2};
        const double w2 = 0.13239415278851, w3 = 0.12593918054483;
        const double w[7] = {0.225, w2, w2, w2, w3, w3, w3};
        q->n = 7;
        for (int i = 0; i < 7; i++) q->l1[i] = l1[i], q->l2[i] = l2[i], q->w[i] = w[i];
        return true;
    }
    if (order == 13) {
        const double a = 0.260345966079038, b = 0.479308067841923;
        const double c = 0.065130102902216, d = 0.869739794195568;
        const double e = 0.048690315425316, f = 0.312865496004875, g = 0.638444188569809;
        const double l1[13] = {1.0 / 3, a, a, b, c, c, d, e, f, g, f, e, g};
        const double l2[13] = {1.0 / 3, a, b, a, c, d, c, f, e, f, g, g, e};
        const double wa = 0.175615257433204, wb = 0.053347235608839, wc = 0.077113760890257;
        const double w[13] = {-0.149570044467670, wa, wa, wa, wb, wb, wb, wc, wc, wc, wc, wc, wc};
        q->n = 13;
        for (int i = 0; i < 13; i++) q->l1[i] = l1[i], q->l2[i] = l2[i], q->w[i] = w[i];
        return true;
    }
    return false;
}

// Gauss-Legendre by Newton from the Tricomi guess -- orient.cpp:39-70.
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    auto legendre = [n](double t, double* pn, double* pn1) {
        double p0 = 1.0, p1 = t;
        for (int j = 2; j <= n; j++) {
            double p2 = ((2 * j - 1) * t * p1 - (j - 1) * p0) / j;
            p0 = p1;
            p1 = p2;
        }
        *pn = p1;
        *pn1 = p0;
    };
    for (int i = 0; i < n; i++) {
        double t = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; it++) {
            double pn, pn1;
            legendre(t, &pn, &pn1);
            double dp = n * (t * pn - pn1) / (t * t - 1.0);
            double dt = -pn / dp;
            t += dt;
            if (std::fabs(dt) < 1e-15) break;
        }
        double pn, pn1;
        legendre(t, &pn, &pn1);
        double dp = n * (t * pn - pn1) / (t * t - 1.0);
        x[i] = t;
        w[i] = 2.0 / ((1.0 - t * t) * dp * dp);
    }
}

// R = Rz(a) Ry(b) Rz(g) -- orient.cpp:4-36; returns R^T row-major.
static void euler_RT(double a, double b, double g, double* RT) {
    double ca = std::cos(a), sa = std::sin(a), cb = std::cos(b), sb = std::sin(b);
    double cg = std::cos(g), sg = std::sin(g);
    double Rz1[3][3] = {{ca, -sa, 0}, {sa, ca, 0}, {0, 0, 1}};
    double Ry[3][3] = {{cb, 0, sb}, {0, 1, 0}, {-sb, 0, cb}};
    double Rz2[3][3] = {{cg, -sg, 0}, {sg, cg, 0}, {0, 0, 1}};
    double R[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            R[i][j] = 0;
            for (int k = 0; k < 3; k++) {
                double t = 0;
                for (int l = 0; l < 3; l++) t += Ry[k][l] * Rz2[l][j];
                R[i][j] += Rz1[i][k] * t;
            }
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) RT[3 * i + j] = R[j][i];
}

// generate_orientations + sort_orientations_nearest -- orient.cpp:73-163.
void orientations(int na, int nb, int ng, int bsym, int gsym, bool mirror, bool sort,
                  std::vector<double>& RT, std::vector<double>& w) {
    std::vector<double> mu, mw;
    if (bsym == 2) {
        std::vector<double> fx, fw;
        gauss_legendre(2 * nb, fx, fw);
        for (int i = 0; i < 2 * nb; i++)
            if (fx[i] > 0) {
                mu.push_back(fx[i]);
                mw.push_back(fw[i] * 2.0);
            }
    } else {
        gauss_legendre(nb, mu, mw);
    }
    double da = 2.0 * M_PI / na, dg = 2.0 * M_PI / ng;
    int eff = mirror ? gsym * 2 : gsym;
    double gstep = 2.0 * M_PI / (eff * ng);
    RT.clear();
    w.clear();
    for (int ia = 0; ia < na; ia++)
        for (int ib = 0; ib < (int)mu.size(); ib++)
            for (int ig = 0; ig < ng; ig++) {
                double g = mirror ? (ig + 0.5) * gstep : ig * gstep;
                double rt[9];
                euler_RT(ia * da, std::acos(mu[ib]), g, rt);
                RT.insert(RT.end(), rt, rt + 9);
                w.push_back(da * mw[ib] * dg / (8.0 * M_PI * M_PI));
            }
    int n = (int)w.size();
    if (!sort || n <= 2) return;
    // greedy nearest neighbour in Frobenius distance, from orientation 0
    std::vector<char> used(n, 0);
    std::vector<int> order;
    order.push_back(0);
    used[0] = 1;
    for (int s = 1; s < n; s++) {
        const double* prev = &RT[9 * order.back()];
        int best = -1;
        double bd = 1e30;
        for (int j = 0; j < n; j++) {
            if (used[j]) continue;
            double d = 0;
            for (int k = 0; k < 9; k++) {
                double df = prev[k] - RT[9 * j + k];
                d += df * df;
            }
            if (d < bd) {
                bd = d;
                best = j;
            }
        }
        order.push_back(best);
        used[best] = 1;
    }
    std::vector<double> RT2(RT.size()), w2(n);
    for (int i = 0; i < n; i++) {
        std::memcpy(&RT2[9 * i], &RT[9 * order[i]], 9 * sizeof(double));
        w2[i] = w[order[i]];
    }
    RT.swap(RT2);
    w.swap(w2);
}

}  // namespace bem

// ------------------------------------------------------------ C ABI (host)
using namespace bem;

static int copy_mesh(const HostMesh& m, int* nv, int* nt, double* verts, int* tris) {
    if (!nv || !nt) return BEM_ERR_INVALID;
    *nv = m.nv();
    *nt = m.nt();
    if (verts)
        for (int i = 0; i < m.nv(); i++) {
            verts[3 * i] = m.verts[i].x;
            verts[3 * i + 1] = m.verts[i].y;
            verts[3 * i + 2] = m.verts[i].z;
        }
    if (tris) std::memcpy(tris, m.tris.data(), m.tris.size() * sizeof(int));
    return BEM_OK;
}

static bool to_mesh(const double* verts, int nv, const int* tris, int nt, HostMesh* m) {
    if (!verts || !tris || nv < 3 || nt < 1) return false;
    m->verts.resize(nv);
    for (int i = 0; i < nv; i++) m->verts[i] = {verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]};
    m->tris.assign(tris, tris + 3 * (size_t)nt);
    for (int v : m->tris)
        if (v < 0 || v >= nv) return false;
    return true;
}

namespace bem {
bool host_mesh_from(const double* verts, int nv, const int* tris, int nt, HostMesh* m) {
    return to_mesh(verts, nv, tris, nt, m);
}
}  // namespace bem

extern "C" {

int bem_mesh_icosphere(double radius, int refinements, int* nv, int* nt, double* verts,
                       int* tris) {
    if (refinements < 0 || refinements > 8 || !(radius > 0)) return BEM_ERR_INVALID;
    return copy_mesh(make_icosphere(radius, refinements), nv, nt, verts, tris);
}

int bem_mesh_hex_prism(double ar, int refinements, int* nv, int* nt, double* verts, int* tris) {
    if (refinements < 0 || refinements > 8 || !(ar > 0)) return BEM_ERR_INVALID;
    return copy_mesh(make_hex_prism(ar, refinements), nv, nt, verts, tris);
}

int bem_mesh_subdivide_flat(const double* verts, int nv, const int* tris, int nt, int* nv_out,
                            int* nt_out, double* verts_out, int* tris_out) {
    HostMesh m;
    if (!to_mesh(verts, nv, tris, nt, &m)) return BEM_ERR_INVALID;
    return copy_mesh(subdivide_flat(m), nv_out, nt_out, verts_out, tris_out);
}

// load_obj -- mesh.cpp:156-250: "v x y z" and "f a b c ..." (fan-triangulated,
// 1-based, "a/b/c" tokens); triangles with a repeated vertex or area < 1e-10
// are removed.
int bem_mesh_load_obj(const char* filename, int* nv, int* nt, double* verts, int* tris,
                      int* n_degenerate, int* n_nonmanifold) {
    if (!filename || !nv || !nt) return BEM_ERR_INVALID;
    std::ifstream f(filename);
    if (!f.is_open()) return BEM_ERR_INVALID;
    HostMesh m;
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        std::string tag;
        is >> tag;
        if (tag == "v") {
            double x, y, z;
            is >> x >> y >> z;
            m.verts.push_back({x, y, z});
        } else if (tag == "f") {
            std::vector<int> fv;
            std::string tok;
            while (is >> tok) fv.push_back(std::atoi(tok.c_str()) - 1);
            for (int i = 1; i + 1 < (int)fv.size(); i++) {
                m.tris.push_back(fv[0]);
                m.tris.push_back(fv[i]);
                m.tris.push_back(fv[i + 1]);
            }
        }
    }
    for (int v : m.tris)
        if (v < 0 || v >= m.nv()) return BEM_ERR_INVALID;
    std::vector<int> keep;
    int ndeg = 0;
    for (int t = 0; t < m.nt(); t++) {
        int a = m.tris[3 * t], b = m.tris[3 * t + 1], c = m.tris[3 * t + 2];
        if (a == b || b == c || a == c) {
            ndeg++;
            continue;
        }
        V3 e1 = sub(m.verts[b], m.verts[a]), e2 = sub(m.verts[c], m.verts[a]);
        if (0.5 * norm(cross(e1, e2)) < 1e-10) {
            ndeg++;
            continue;
        }
        keep.push_back(a);
        keep.push_back(b);
        keep.push_back(c);
    }
    m.tris.swap(keep);
    std::map<std::pair<int, int>, int> cnt;
    for (int t = 0; t < m.nt(); t++)
        for (int e = 0; e < 3; e++) {
            int a = m.tris[3 * t + e], b = m.tris[3 * t + (e + 1) % 3];
            cnt[{std::min(a, b), std::max(a, b)}]++;
        }
    int nm = 0;
    for (auto& kv : cnt) nm += kv.second > 2;
    if (n_degenerate) *n_degenerate = ndeg;
    if (n_nonmanifold) *n_nonmanifold = nm;
    return copy_mesh(m, nv, nt, verts, tris);
}

// mesh_volume -- mesh.cpp:252-261
double bem_mesh_volume(const double* verts, int nv, const int* tris, int nt) {
    (void)nv;
    double vol = 0;
    for (int t = 0; t < nt; t++) {
        const double* a = verts + 3 * tris[3 * t];
        const double* b = verts + 3 * tris[3 * t + 1];
        const double* c = verts + 3 * tris[3 * t + 2];
        V3 bc = cross({b[0], b[1], b[2]}, {c[0], c[1], c[2]});
        vol += a[0] * bc.x + a[1] * bc.y + a[2] * bc.z;
    }
    return vol / 6.0;
}

// normalize_mesh -- mesh.cpp:263-283 (bounding-sphere radius when the volume
// vanishes)
int bem_mesh_normalize(double* verts, int nv, const int* tris, int nt, double* a_eq_out) {
    if (!verts || !tris || nv < 1) return BEM_ERR_INVALID;
    double vol = std::fabs(bem_mesh_volume(verts, nv, tris, nt));
    double a_eq = std::cbrt(3.0 * vol / (4.0 * M_PI));
    if (a_eq < 1e-30) {
        double c[3] = {0, 0, 0}, r2 = 0;
        for (int i = 0; i < nv; i++)
            for (int d = 0; d < 3; d++) c[d] += verts[3 * i + d];
        for (int d = 0; d < 3; d++) c[d] /= nv;
        for (int i = 0; i < nv; i++) {
            double s = 0;
            for (int d = 0; d < 3; d++) s += (verts[3 * i + d] - c[d]) * (verts[3 * i + d] - c[d]);
            r2 = std::max(r2, s);
        }
        a_eq = std::sqrt(r2);
    }
    double s = 1.0 / a_eq;
    for (int i = 0; i < 3 * nv; i++) verts[i] *= s;
    if (a_eq_out) *a_eq_out = a_eq;
    return BEM_OK;
}

// mesh_dmax -- mesh.cpp:285-294 (bounding-box diagonal)
double bem_mesh_dmax(const double* verts, int nv) {
    double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
    for (int i = 0; i < nv; i++)
        for (int d = 0; d < 3; d++) {
            lo[d] = std::min(lo[d], verts[3 * i + d]);
            hi[d] = std::max(hi[d], verts[3 * i + d]);
        }
    double s = 0;
    for (int d = 0; d < 3; d++) s += (hi[d] - lo[d]) * (hi[d] - lo[d]);
    return std::sqrt(s);
}

int bem_rwg_build(const double* verts, int nv, const int* tris, int nt, int* N, int* tri_p,
                  int* tri_m, double* free_p, double* free_m, double* length, double* area_p,
                  double* area_m) {
    HostMesh m;
    if (!N || !to_mesh(verts, nv, tris, nt, &m)) return BEM_ERR_INVALID;
    HostRWG r = build_rwg(m);
    *N = r.N;
    for (int n = 0; n < r.N; n++) {
        if (tri_p) tri_p[n] = r.tri_p[n];
        if (tri_m) tri_m[n] = r.tri_m[n];
        if (free_p) free_p[3 * n] = r.free_p[n].x, free_p[3 * n + 1] = r.free_p[n].y, free_p[3 * n + 2] = r.free_p[n].z;
        if (free_m) free_m[3 * n] = r.free_m[n].x, free_m[3 * n + 1] = r.free_m[n].y, free_m[3 * n + 2] = r.free_m[n].z;
        if (length) length[n] = r.length[n];
        if (area_p) area_p[n] = r.area_p[n];
        if (area_m) area_m[n] = r.area_m[n];
    }
    return BEM_OK;
}

int bem_tri_quadrature(int order, int* npts, double* pts, double* wts) {
    Quad q;
    if (!npts || !quadrature(order, &q)) return BEM_ERR_INVALID;
    *npts = q.n;
    for (int i = 0; i < q.n; i++) {
        if (pts) pts[2 * i] = q.l1[i], pts[2 * i + 1] = q.l2[i];
        if (wts) wts[i] = q.w[i];
    }
    return BEM_OK;
}

int bem_orientations(int na, int nb, int ng, int bsym, int gsym, int mirror, int sort,
                     int* count, double* RT, double* w) {
    if (!count || na < 1 || nb < 1 || ng < 1 || (bsym != 1 && bsym != 2) || gsym < 1)
        return BEM_ERR_INVALID;
    std::vector<double> rt, ww;
    orientations(na, nb, ng, bsym, gsym, mirror != 0, sort != 0, rt, ww);
    *count = (int)ww.size();
    if (RT) std::memcpy(RT, rt.data(), rt.size() * sizeof(double));
    if (w) std::memcpy(w, ww.data(), ww.size() * sizeof(double));
    return BEM_OK;
}

int bem_gauss_legendre(int n, double* nodes, double* weights) {
    if (n < 1 || !nodes || !weights) return BEM_ERR_INVALID;
    std::vector<double> x, w;
    gauss_legendre(n, x, w);
    std::memcpy(nodes, x.data(), n * sizeof(double));
    std::memcpy(weights, w.data(), n * sizeof(double));
    return BEM_OK;
}

}  // extern "C"
