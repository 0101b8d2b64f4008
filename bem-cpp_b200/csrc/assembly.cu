// PMCHWT assembly on the device (FP64).
//
// Restates assemble_LK_kernel (assembly.cu:14-135), precompute_half
// (assembly.cu:150-201), apply_singular_corrections (assembly.cu:208-321),
// the symmetrisation (assembly.cu:494-502) and the block fill of
// assemble_pmchwt (pmchwt.cu:36-51) as one device pipeline:
//
//   1. graglia_kernel     -- per (triangle, point): Graglia P and the
//                            finite-difference vector potential V (FP64).
//   2. assemble_kernel    -- per 16x16 tile of RWG pairs (m <= n tiles only):
//                            all four half pairs, both media, quadrature part of
//                            L and K, written straight into the four Z blocks and
//                            mirrored (L and K are symmetric).
//   3. singular_fixup     -- per RWG pair sharing a triangle: the symmetrised
//                            same-triangle correction (S[m,n] + S[n,m])/2.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "asm_device.cuh"
#include "bem_internal.h"

namespace bem {


// ------------------------------------------------------------ geometry upload
bool host_mesh_from(const double* verts, int nv, const int* tris, int nt, HostMesh* m);

// Position-dependent geometry arrays (everything the vertex coordinates
// enter): per-half quadrature points, basis values, weights, divergences,
// free vertices; triangle vertices; per-triangle centroid-relative data.
struct PosArrays {
    std::vector<double> px, py, pz, fx, fy, fz, cx, cy, cz, jw, div, coef, frx, fry, frz, tv, tc, tu, tjw, hpi;
    std::vector<int> tri;
};

static void position_arrays(const bem_geom* g, PosArrays& A) {
    const HostMesh& m = g->mesh;
    const HostRWG& r = g->rwg;
    const Quad& q = g->quad;
    const int N = r.N, Nq = q.n, nt = m.nt();
    const size_t P = (size_t)2 * N * Nq;
    auto& px = A.px; auto& py = A.py; auto& pz = A.pz; auto& fx = A.fx; auto& fy = A.fy; auto& fz = A.fz;
    auto& cx = A.cx; auto& cy = A.cy; auto& cz = A.cz; auto& jw = A.jw;
    for (auto* v : {&px, &py, &pz, &fx, &fy, &fz, &cx, &cy, &cz, &jw}) v->assign(P, 0.0);
    auto& div = A.div; auto& coef = A.coef; auto& frx = A.frx; auto& fry = A.fry; auto& frz = A.frz;
    for (auto* v : {&div, &coef, &frx, &fry, &frz}) v->assign(2 * N, 0.0);
    auto& tri = A.tri;
    tri.assign(2 * N, 0);
    for (int h = 0; h < 2; h++) {
        int sign = h == 0 ? 1 : -1;
        for (int n = 0; n < N; n++) {
            int t = h == 0 ? r.tri_p[n] : r.tri_m[n];
            V3 fr = h == 0 ? r.free_p[n] : r.free_m[n];
            double area = h == 0 ? r.area_p[n] : r.area_m[n];
            double c = sign * r.length[n] / (2.0 * area);
            int hn = h * N + n;
            div[hn] = sign * r.length[n] / area;
            coef[hn] = c;
            frx[hn] = fr.x, fry[hn] = fr.y, frz[hn] = fr.z;
            tri[hn] = t;
            V3 v0 = m.verts[m.tris[3 * t]], v1 = m.verts[m.tris[3 * t + 1]],
               v2 = m.verts[m.tris[3 * t + 2]];
            for (int k = 0; k < Nq; k++) {
                double l1 = q.l1[k], l2 = q.l2[k], l0 = 1.0 - l1 - l2;
                // r = v0 l0 + v1 l1 + v2 l2, evaluated left to right as the reference
                double rx = (v0.x * l0 + v1.x * l1) + v2.x * l2;
                double ry = (v0.y * l0 + v1.y * l1) + v2.y * l2;
                double rz = (v0.z * l0 + v1.z * l1) + v2.z * l2;
                double ffx = (rx - fr.x) * c, ffy = (ry - fr.y) * c, ffz = (rz - fr.z) * c;
                size_t i = (size_t)hn * Nq + k;
                px[i] = rx, py[i] = ry, pz[i] = rz;
                fx[i] = ffx, fy[i] = ffy, fz[i] = ffz;
                cx[i] = ffy * rz - ffz * ry;
                cy[i] = ffz * rx - ffx * rz;
                cz[i] = ffx * ry - ffy * rx;
                jw[i] = area * q.w[k];
            }
        }
    }
    auto& tv = A.tv;
    tv.assign(9 * (size_t)nt, 0.0);
    for (int t = 0; t < nt; t++)
        for (int j = 0; j < 3; j++) {
            V3 v = m.verts[m.tris[3 * t + j]];
            tv[9 * t + 3 * j] = v.x, tv[9 * t + 3 * j + 1] = v.y, tv[9 * t + 3 * j + 2] = v.z;
        }
    // triangle-pair assembly data: per triangle the centroid, the quadrature
    // points relative to it (the same points as the halves') and area x
    // weight; per half the free vertex relative to its triangle's centroid
    auto& tc = A.tc; auto& tu = A.tu; auto& tjw = A.tjw; auto& hpi = A.hpi;
    tc.assign(3 * (size_t)nt, 0.0);
    tu.assign(3 * (size_t)nt * Nq, 0.0);
    tjw.assign((size_t)nt * Nq, 0.0);
    hpi.assign(3 * (size_t)2 * N, 0.0);
    std::vector<double> tarea(nt, -1.0);
    for (int h = 0; h < 2; h++)
        for (int n = 0; n < N; n++) {
            const int t = h == 0 ? r.tri_p[n] : r.tri_m[n];
            if (tarea[t] < 0) tarea[t] = h == 0 ? r.area_p[n] : r.area_m[n];
        }
    for (int t = 0; t < nt; t++) {
        V3 v0 = m.verts[m.tris[3 * t]], v1 = m.verts[m.tris[3 * t + 1]], v2 = m.verts[m.tris[3 * t + 2]];
        const double cx0 = (v0.x + v1.x + v2.x) / 3.0, cy0 = (v0.y + v1.y + v2.y) / 3.0,
                     cz0 = (v0.z + v1.z + v2.z) / 3.0;
        tc[3 * t] = cx0, tc[3 * t + 1] = cy0, tc[3 * t + 2] = cz0;
        for (int k = 0; k < Nq; k++) {
            double l1 = q.l1[k], l2 = q.l2[k], l0 = 1.0 - l1 - l2;
            double rx = (v0.x * l0 + v1.x * l1) + v2.x * l2;
            double ry = (v0.y * l0 + v1.y * l1) + v2.y * l2;
            double rz = (v0.z * l0 + v1.z * l1) + v2.z * l2;
            size_t i = ((size_t)t * Nq + k) * 3;
            tu[i] = rx - cx0, tu[i + 1] = ry - cy0, tu[i + 2] = rz - cz0;
            tjw[(size_t)t * Nq + k] = (tarea[t] > 0 ? tarea[t] : 0.0) * q.w[k];
        }
    }
    for (int h = 0; h < 2; h++)
        for (int n = 0; n < N; n++) {
            const int t = h == 0 ? r.tri_p[n] : r.tri_m[n];
            const V3 fr = h == 0 ? r.free_p[n] : r.free_m[n];
            size_t i = ((size_t)h * N + n) * 3;
            hpi[i] = fr.x - tc[3 * t], hpi[i + 1] = fr.y - tc[3 * t + 1], hpi[i + 2] = fr.z - tc[3 * t + 2];
        }
}

int geom_upload(bem_ctx* ctx, bem_geom* g) {
    const HostMesh& m = g->mesh;
    const HostRWG& r = g->rwg;
    const Quad& q = g->quad;
    const int N = r.N, Nq = q.n, nt = m.nt();
    const size_t P = (size_t)2 * N * Nq;
    PosArrays A;
    position_arrays(g, A);
    auto& px = A.px; auto& py = A.py; auto& pz = A.pz; auto& fx = A.fx; auto& fy = A.fy; auto& fz = A.fz;
    auto& cx = A.cx; auto& cy = A.cy; auto& cz = A.cz; auto& jw = A.jw;
    auto& div = A.div; auto& coef = A.coef; auto& frx = A.frx; auto& fry = A.fry; auto& frz = A.frz;
    auto& tri = A.tri; auto& tv = A.tv; auto& tc = A.tc; auto& tu = A.tu; auto& tjw = A.tjw; auto& hpi = A.hpi;
    // singular pairs: halves per triangle, ordered (test, source) items per
    // unordered RWG pair
    std::vector<std::vector<int>> on_tri(nt);
    for (int h = 0; h < 2; h++)
        for (int n = 0; n < N; n++) on_tri[h == 0 ? r.tri_p[n] : r.tri_m[n]].push_back(h * N + n);
    std::map<std::pair<int, int>, std::vector<int>> slot;  // (m<=n) -> items (t, a, b)
    for (int t = 0; t < nt; t++)
        for (int a : on_tri[t])
            for (int b : on_tri[t]) {
                int mm = a % N, nn = b % N;
                auto& v = slot[{std::min(mm, nn), std::max(mm, nn)}];
                v.push_back(t);
                v.push_back(a);
                v.push_back(b);
            }
    std::vector<int> pair_mn, item_ptr{0}, item;
    for (auto& kv : slot) {
        pair_mn.push_back(kv.first.first);
        pair_mn.push_back(kv.first.second);
        item.insert(item.end(), kv.second.begin(), kv.second.end());
        item_ptr.push_back((int)item.size() / 3);
    }
    g->sing.npairs = (int)pair_mn.size() / 2;
    g->sing.nitems = (int)item.size() / 3;

    // RWGs in the Morton order of their triangles' centroids: each triangle
    // in turn appends its RWGs not placed yet, so a tile of 16 consecutive
    // RWGs touches ~17 distinct triangles instead of ~21-32
    std::vector<int> torder(nt);
    {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int t = 0; t < nt; t++)
            for (int j = 0; j < 3; j++) lo[j] = std::min(lo[j], tc[3 * t + j]), hi[j] = std::max(hi[j], tc[3 * t + j]);
        const double span = std::max(std::max(hi[0] - lo[0], hi[1] - lo[1]), std::max(hi[2] - lo[2], 1e-300));
        std::vector<uint64_t> key(nt);
        for (int t = 0; t < nt; t++) {
            uint64_t code = 0;
            uint64_t c3[3];
            for (int j = 0; j < 3; j++) {
                double f = (tc[3 * t + j] - lo[j]) / span;
                c3[j] = (uint64_t)std::min(2097151.0, std::max(0.0, f * 2097151.0));
            }
            for (int b = 20; b >= 0; b--)
                for (int j = 0; j < 3; j++) code = (code << 1) | ((c3[j] >> b) & 1u);
            key[t] = code;
        }
        for (int t = 0; t < nt; t++) torder[t] = t;
        std::stable_sort(torder.begin(), torder.end(), [&](int x, int y) { return key[x] < key[y]; });
    }
    std::vector<int> tri_half(3 * (size_t)nt, -1);
    for (int h = 0; h < 2; h++)
        for (int n = 0; n < N; n++) {
            const int t = h == 0 ? r.tri_p[n] : r.tri_m[n];
            int j = 0;
            while (j < 3 && tri_half[3 * (size_t)t + j] >= 0) j++;
            if (j == 3) return fail(ctx, BEM_ERR_INVALID, "triangle %d carries more than 3 RWG halves", t);
            tri_half[3 * (size_t)t + j] = h * N + n;
        }
    std::vector<std::vector<int>> rwg_of_tri(nt);
    for (int n = 0; n < N; n++) rwg_of_tri[r.tri_p[n]].push_back(n), rwg_of_tri[r.tri_m[n]].push_back(n);
    const int ntile = (N + ASM_TILE - 1) / ASM_TILE;
    std::vector<int> perm, pos(N, -1);
    perm.reserve(N);
    for (int t : torder)
        for (int n : rwg_of_tri[t])
            if (pos[n] < 0) pos[n] = (int)perm.size(), perm.push_back(n);
    std::vector<int> tile_rwg((size_t)ntile * ASM_TILE, -1), tile_tri((size_t)ntile * ASM_TRI_MAX, -1), tile_ntri(ntile, 0);
    std::vector<unsigned char> tile_ent((size_t)ntile * ASM_TRI_MAX * 3, 0xff);
    for (int tl = 0; tl < ntile; tl++) {
        int cnt = 0;
        for (int sl = 0; sl < ASM_TILE && tl * ASM_TILE + sl < N; sl++) {
            const int n = perm[tl * ASM_TILE + sl];
            tile_rwg[(size_t)tl * ASM_TILE + sl] = n;
            for (int h = 0; h < 2; h++) {
                const int t = h == 0 ? r.tri_p[n] : r.tri_m[n];
                int li = 0;
                while (li < cnt && tile_tri[(size_t)tl * ASM_TRI_MAX + li] != t) li++;
                if (li == cnt) tile_tri[(size_t)tl * ASM_TRI_MAX + cnt++] = t;
                unsigned char* e = &tile_ent[((size_t)tl * ASM_TRI_MAX + li) * 3];
                int j = 0;
                while (j < 3 && e[j] != 0xff) j++;
                if (j == 3) return fail(ctx, BEM_ERR_INVALID, "triangle %d carries more than 3 RWG halves", t);
                e[j] = (unsigned char)(sl * 2 + h);
            }
        }
        tile_ntri[tl] = cnt;
    }

    // one device allocation, 256-byte aligned sub-arrays
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (bytes + 255) & ~(size_t)255;
        return o;
    };
    size_t o_pt[10];
    for (int i = 0; i < 10; i++) o_pt[i] = take(P * 8);
    size_t o_div = take(2 * N * 8), o_coef = take(2 * N * 8), o_fr = take(3 * 2 * N * 8);
    size_t o_tri = take(2 * N * 4);
    size_t o_pmn = take(pair_mn.size() * 4), o_iptr = take(item_ptr.size() * 4),
           o_item = take(item.size() * 4);
    size_t o_P = take((size_t)nt * Nq * 8), o_V = take((size_t)nt * Nq * 3 * 8),
           o_tv = take(tv.size() * 8);
    size_t o_tc = take(tc.size() * 8), o_tu = take(tu.size() * 8), o_tjw = take(tjw.size() * 8),
           o_hpi = take(hpi.size() * 8), o_trwg = take(tile_rwg.size() * 4), o_pos = take((size_t)N * 4),
           o_ttri = take(tile_tri.size() * 4), o_tntri = take((size_t)ntile * 4), o_tent = take(tile_ent.size()),
           o_tflag = take((size_t)ntile), o_rrec = take((size_t)N), o_thalf = take(tri_half.size() * 4);
    g->dmem = devmem_alloc(ctx->device, off, ctx);
    if (!g->dmem) return fail(ctx, BEM_ERR_OOM, "geometry arrays (%zu bytes)", off);
    g->dmem_bytes = off;
    char* base = (char*)g->dmem;
    double** pts[10] = {&g->half.px, &g->half.py, &g->half.pz, &g->half.fx, &g->half.fy,
                        &g->half.fz, &g->half.cx, &g->half.cy, &g->half.cz, &g->half.jw};
    std::vector<double>* src[10] = {&px, &py, &pz, &fx, &fy, &fz, &cx, &cy, &cz, &jw};
    for (int i = 0; i < 10; i++) {
        *pts[i] = (double*)(base + o_pt[i]);
        BEM_TRY(h2d(ctx, *pts[i], src[i]->data(), P * 8));
    }
    g->half.div = (double*)(base + o_div);
    g->half.tri = (int*)(base + o_tri);
    double* d_coef = (double*)(base + o_coef);
    double* d_fr = (double*)(base + o_fr);
    BEM_TRY(h2d(ctx, g->half.div, div.data(), 2 * N * 8));
    BEM_TRY(h2d(ctx, d_coef, coef.data(), 2 * N * 8));
    BEM_TRY(h2d(ctx, d_fr, frx.data(), 2 * N * 8));
    BEM_TRY(h2d(ctx, d_fr + 2 * N, fry.data(), 2 * N * 8));
    BEM_TRY(h2d(ctx, d_fr + 4 * N, frz.data(), 2 * N * 8));
    BEM_TRY(h2d(ctx, g->half.tri, tri.data(), 2 * N * 4));
    g->sing.pair_mn = (int*)(base + o_pmn);
    g->sing.item_ptr = (int*)(base + o_iptr);
    g->sing.item = (int*)(base + o_item);
    g->sing.P = (double*)(base + o_P);
    g->sing.V = (double*)(base + o_V);
    g->sing.tv = (double*)(base + o_tv);
    BEM_TRY(h2d(ctx, g->sing.pair_mn, pair_mn.data(), pair_mn.size() * 4));
    BEM_TRY(h2d(ctx, g->sing.item_ptr, item_ptr.data(), item_ptr.size() * 4));
    BEM_TRY(h2d(ctx, g->sing.item, item.data(), item.size() * 4));
    BEM_TRY(h2d(ctx, g->sing.tv, tv.data(), tv.size() * 8));
    DevTriAsm& ta = g->tri;
    ta.c = (double*)(base + o_tc);
    ta.u = (double*)(base + o_tu);
    ta.jw = (double*)(base + o_tjw);
    ta.pi = (double*)(base + o_hpi);
    ta.tile_rwg = (int*)(base + o_trwg);
    ta.pos = (int*)(base + o_pos);
    ta.tile_tri = (int*)(base + o_ttri);
    ta.tile_ntri = (int*)(base + o_tntri);
    ta.tile_ent = (unsigned char*)(base + o_tent);
    ta.tile_flag = (unsigned char*)(base + o_tflag);
    ta.rwg_rec = (unsigned char*)(base + o_rrec);
    ta.ntile = ntile;
    ta.tri_half = (int*)(base + o_thalf);
    BEM_TRY(h2d(ctx, ta.tri_half, tri_half.data(), tri_half.size() * 4));
    BEM_TRY(h2d(ctx, ta.c, tc.data(), tc.size() * 8));
    BEM_TRY(h2d(ctx, ta.u, tu.data(), tu.size() * 8));
    BEM_TRY(h2d(ctx, ta.jw, tjw.data(), tjw.size() * 8));
    BEM_TRY(h2d(ctx, ta.pi, hpi.data(), hpi.size() * 8));
    BEM_TRY(h2d(ctx, ta.tile_rwg, tile_rwg.data(), tile_rwg.size() * 4));
    BEM_TRY(h2d(ctx, ta.pos, pos.data(), (size_t)N * 4));
    BEM_TRY(h2d(ctx, ta.tile_tri, tile_tri.data(), tile_tri.size() * 4));
    BEM_TRY(h2d(ctx, ta.tile_ntri, tile_ntri.data(), (size_t)ntile * 4));
    BEM_TRY(h2d(ctx, ta.tile_ent, tile_ent.data(), tile_ent.size()));
    // half coefficient and free vertex live right after div (see fixup kernel)
    (void)d_coef;
    (void)d_fr;
    g->sing_coef = d_coef;
    g->sing_free = d_fr;
    return BEM_OK;
}

int geom_set_vertices(bem_ctx* ctx, bem_geom* g, const double* verts) {
    HostRWG& r = g->rwg;
    HostMesh& m = g->mesh;
    if (!verts || r.edge_lo.size() != (size_t)r.N || r.vfree_p.size() != (size_t)r.N)
        return fail(ctx, BEM_ERR_INVALID, "vertex update needs a geometry built from its mesh");
    for (int i = 0; i < m.nv(); i++) m.verts[i] = {verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]};
    rwg_refresh(m, r);
    PosArrays A;
    position_arrays(g, A);
    const int N = r.N;
    const size_t P = A.px.size();
    cudaStream_t st = ctx->stream;
    double* dst[10] = {g->half.px, g->half.py, g->half.pz, g->half.fx, g->half.fy,
                       g->half.fz, g->half.cx, g->half.cy, g->half.cz, g->half.jw};
    const std::vector<double>* src[10] = {&A.px, &A.py, &A.pz, &A.fx, &A.fy, &A.fz, &A.cx, &A.cy, &A.cz, &A.jw};
    for (int i = 0; i < 10; i++)
        BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dst[i], src[i]->data(), P * 8, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(g->half.div, A.div.data(), 2 * (size_t)N * 8, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(g->sing_coef, A.coef.data(), 2 * (size_t)N * 8, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(g->sing_free, A.frx.data(), 2 * (size_t)N * 8, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(g->sing_free + 2 * N, A.fry.data(), 2 * (size_t)N * 8, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(g->sing_free + 4 * N, A.frz.data(), 2 * (size_t)N * 8, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(g->sing.tv, A.tv.data(), A.tv.size() * 8, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(g->tri.c, A.tc.data(), A.tc.size() * 8, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(g->tri.u, A.tu.data(), A.tu.size() * 8, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(g->tri.jw, A.tjw.data(), A.tjw.size() * 8, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(g->tri.pi, A.hpi.data(), A.hpi.size() * 8, cudaMemcpyHostToDevice, st));
    return BEM_OK;
}

// One thread per (triangle, point): P and V = r P - grad W (central
// differences, eps = 1e-6) -- graglia.h:90-112.
__global__ void graglia_kernel(const double* __restrict__ tv, int nt, TriQ q,
                               double* __restrict__ P, double* __restrict__ V) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt * q.n) return;
    int t = i / q.n, k = i % q.n;
    double v[9];
    for (int j = 0; j < 9; j++) v[j] = tv[9 * t + j];
    graglia_point(v, q.l1[k], q.l2[k], q, &P[i], &V[3 * i]);
}

// ------------------------------------------------------------ main assembly
constexpr int TILE = 16;
static_assert(TILE == ASM_TILE, "assembly band width");
constexpr int MAXQ = 13;

struct AsmArgs {
    DevHalf h;
    int N, Nq;
    int ntile;       // tiles per side
    Medium med[2];   // ext, int (only med[0] when nmed == 1)
    double eta_e, eta_i;
    unsigned flags;
    // outputs
    double2* Z;      // row-major 2N x 2N: PMCHWT (nmed == 2) or A_ext (nmed == 1)
    int64_t ldz;
    double2* L;      // row-major N x N (nmed == 1, Z null)
    double2* K;
    int64_t ld;
    // optional: only tile pairs with a flagged row or column tile are computed
    const unsigned char* tile_flag;
    const double* coef;  // (2N) sign*l/(2A) per half (triangle-pair kernel)
};

template <int NMED>
__global__ void __launch_bounds__(256) assemble_kernel(AsmArgs a) {
    // upper-triangular tile index -> (tile row bi, tile col bj), bi <= bj
    int64_t lin = blockIdx.x;
    int T = a.ntile;
    // row bi starts at offset bi*T - bi*(bi-1)/2
    int bi = (int)floor((2.0 * T + 1.0 - sqrt((2.0 * T + 1.0) * (2.0 * T + 1.0) - 8.0 * (double)lin)) * 0.5);
    if (bi < 0) bi = 0;
    while (bi > 0 && (int64_t)bi * T - (int64_t)bi * (bi - 1) / 2 > lin) bi--;
    while ((int64_t)(bi + 1) * T - (int64_t)(bi + 1) * bi / 2 <= lin) bi++;
    int bj = bi + (int)(lin - ((int64_t)bi * T - (int64_t)bi * (bi - 1) / 2));

    const int N = a.N, Nq = a.Nq;
    const int tx = threadIdx.x % TILE, ty = threadIdx.x / TILE;
    if (a.tile_flag && !a.tile_flag[bi] && !a.tile_flag[bj]) return;  // a tile the caller keeps
    const int m0 = bi * TILE, n0 = bj * TILE;

    // source data of the tile's columns: [half][q][col]
    __shared__ double s_px[2][MAXQ][TILE], s_py[2][MAXQ][TILE], s_pz[2][MAXQ][TILE];
    __shared__ double s_fx[2][MAXQ][TILE], s_fy[2][MAXQ][TILE], s_fz[2][MAXQ][TILE];
    __shared__ double s_cx[2][MAXQ][TILE], s_cy[2][MAXQ][TILE], s_cz[2][MAXQ][TILE];
    __shared__ double s_jw[2][MAXQ][TILE];
    __shared__ double s_div[2][TILE];
    __shared__ int s_tri[2][TILE];
    for (int i = threadIdx.x; i < 2 * Nq * TILE; i += blockDim.x) {
        int col = i % TILE, q = (i / TILE) % Nq, h = i / (TILE * Nq);
        int n = min(n0 + col, N - 1);
        size_t p = ((size_t)(h * N + n)) * Nq + q;
        s_px[h][q][col] = a.h.px[p];
        s_py[h][q][col] = a.h.py[p];
        s_pz[h][q][col] = a.h.pz[p];
        s_fx[h][q][col] = a.h.fx[p];
        s_fy[h][q][col] = a.h.fy[p];
        s_fz[h][q][col] = a.h.fz[p];
        s_cx[h][q][col] = a.h.cx[p];
        s_cy[h][q][col] = a.h.cy[p];
        s_cz[h][q][col] = a.h.cz[p];
        s_jw[h][q][col] = a.h.jw[p];
    }
    if (threadIdx.x < 2 * TILE) {
        int h = threadIdx.x / TILE, col = threadIdx.x % TILE;
        int n = min(n0 + col, N - 1);
        s_div[h][col] = a.h.div[h * N + n];
        s_tri[h][col] = a.h.tri[h * N + n];
    }
    __syncthreads();

    const int m = min(m0 + ty, N - 1);
    const bool exact = (a.flags & BEM_ASM_GSMOOTH_EXACT) != 0;
    cplx Lv[NMED], Ls[NMED], Kk[NMED];
    for (int e = 0; e < NMED; e++) Lv[e] = Ls[e] = Kk[e] = {0.0, 0.0};

    for (int th = 0; th < 2; th++) {
        const int thn = th * N + m;
        const int ttri = a.h.tri[thn];
        const double tdiv = a.h.div[thn];
        for (int sh = 0; sh < 2; sh++) {
            const bool sing = (ttri == s_tri[sh][tx]);
            const double dd = tdiv * s_div[sh][tx];
            cplx Lsb[NMED];
            for (int e = 0; e < NMED; e++) Lsb[e] = {0.0, 0.0};
            for (int q = 0; q < Nq; q++) {
                size_t tp = (size_t)thn * Nq + q;
                const double tpx = a.h.px[tp], tpy = a.h.py[tp], tpz = a.h.pz[tp];
                const double tfx = a.h.fx[tp], tfy = a.h.fy[tp], tfz = a.h.fz[tp];
                const double tcx = a.h.cx[tp], tcy = a.h.cy[tp], tcz = a.h.cz[tp];
                const double tjw = a.h.jw[tp];
                for (int qs = 0; qs < Nq; qs++) {
                    double dx = tpx - s_px[sh][qs][tx];
                    double dy = tpy - s_py[sh][qs][tx];
                    double dz = tpz - s_pz[sh][qs][tx];
                    double R = sqrt(dx * dx + dy * dy + dz * dz);
                    double Rs = fmax(R, 1e-15);
                    double invR = 1.0 / Rs;
                    // rounded on its own: the literal G_smooth subtracts it
                    // from G, and a multiply-add fused across the two would
                    // leave its rounding error (~0.01 at R_s = 1e-15)
                    double i4R = __dmul_rn(INV4PI_D, invR);
                    double jwp = tjw * s_jw[sh][qs][tx];
                    double fdot = tfx * s_fx[sh][qs][tx] + tfy * s_fy[sh][qs][tx] + tfz * s_fz[sh][qs][tx];
                    // f_t . ((r_t - r_s) x f_s) = (f_t x r_t).f_s + f_t.(f_s x r_s)
                    double trip = (tcx * s_fx[sh][qs][tx] + tcy * s_fy[sh][qs][tx] + tcz * s_fz[sh][qs][tx]) +
                                  (tfx * s_cx[sh][qs][tx] + tfy * s_cy[sh][qs][tx] + tfz * s_cz[sh][qs][tx]);
                    bool kval = !sing && R > 1e-12;
#pragma unroll
                    for (int e = 0; e < NMED; e++) {
                        const Medium k = a.med[e];
                        double s, c;
                        sincos(k.kr * Rs, &s, &c);
                        double ea = (k.ki != 0.0) ? exp_decay(k.ki * Rs) : 1.0;
                        cplx G = {ea * c * i4R, ea * s * i4R};
                        cplx Gu = G;
                        if (sing) {
                            if (exact) Gu = g_smooth_exact(k, R);
                            else Gu.re -= i4R;
                        }
                        cplx Gj = {Gu.re * jwp, Gu.im * jwp};
                        Lv[e].re += fdot * Gj.re;
                        Lv[e].im += fdot * Gj.im;
                        Lsb[e].re += Gj.re;
                        Lsb[e].im += Gj.im;
                        if (kval) {
                            // grad G coefficient (ik - 1/R)/R
                            cplx gc = cmul(G, cplx{(-k.ki - invR) * invR, k.kr * invR});
                            double w = jwp * trip;
                            Kk[e].re += gc.re * w;
                            Kk[e].im += gc.im * w;
                        }
                    }
                }
            }
            for (int e = 0; e < NMED; e++) {
                Ls[e].re += dd * Lsb[e].re;
                Ls[e].im += dd * Lsb[e].im;
            }
        }
    }
    const int n = n0 + tx;
    const int mm = m0 + ty;
    if (mm >= N || n >= N) return;
    // L = ik Lvec - (i/k) sum(div div Lscl)
    cplx Lf[NMED];
    for (int e = 0; e < NMED; e++) {
        Medium k = a.med[e];
        cplx ik = {-k.ki, k.kr};
        double k2 = k.kr * k.kr + k.ki * k.ki;
        cplx iok = {k.ki / k2, k.kr / k2};  // i/k
        cplx t1 = cmul(ik, Lv[e]), t2 = cmul(iok, Ls[e]);
        Lf[e] = {t1.re - t2.re, t1.im - t2.im};
    }
    // L and K are symmetric: in a diagonal tile only the thread of the upper
    // entry writes, to both positions, so the stored blocks are exactly
    // symmetric (as after the reference's (X + X^T)/2, assembly.cu:494-502)
    if (bi == bj && n < mm) return;
    const bool mirror = (n != mm);
    if (a.Z) {
        // PMCHWT blocks; with one medium the exterior-only A_ext
        // [[eta_e L_e, -K_e], [K_e, L_e / eta_e]] (bem_core.py:1071-1090)
        cplx TL, BR, Ks;
        if constexpr (NMED == 2) {
            TL = {a.eta_e * Lf[0].re + a.eta_i * Lf[1].re, a.eta_e * Lf[0].im + a.eta_i * Lf[1].im};
            BR = {Lf[0].re / a.eta_e + Lf[1].re / a.eta_i, Lf[0].im / a.eta_e + Lf[1].im / a.eta_i};
            Ks = {Kk[0].re + Kk[1].re, Kk[0].im + Kk[1].im};
        } else {
            TL = {a.eta_e * Lf[0].re, a.eta_e * Lf[0].im};
            BR = {Lf[0].re / a.eta_e, Lf[0].im / a.eta_e};
            Ks = Kk[0];
        }
        double2* Z = a.Z;
        int64_t ld = a.ldz;
        Z[(int64_t)mm * ld + n] = make_double2(TL.re, TL.im);
        Z[(int64_t)mm * ld + N + n] = make_double2(-Ks.re, -Ks.im);
        Z[(int64_t)(N + mm) * ld + n] = make_double2(Ks.re, Ks.im);
        Z[(int64_t)(N + mm) * ld + N + n] = make_double2(BR.re, BR.im);
        if (mirror) {
            Z[(int64_t)n * ld + mm] = make_double2(TL.re, TL.im);
            Z[(int64_t)n * ld + N + mm] = make_double2(-Ks.re, -Ks.im);
            Z[(int64_t)(N + n) * ld + mm] = make_double2(Ks.re, Ks.im);
            Z[(int64_t)(N + n) * ld + N + mm] = make_double2(BR.re, BR.im);
        }
    } else {
        a.L[(int64_t)mm * a.ld + n] = make_double2(Lf[0].re, Lf[0].im);
        a.K[(int64_t)mm * a.ld + n] = make_double2(Kk[0].re, Kk[0].im);
        if (mirror) {
            a.L[(int64_t)n * a.ld + mm] = make_double2(Lf[0].re, Lf[0].im);
            a.K[(int64_t)n * a.ld + mm] = make_double2(Kk[0].re, Kk[0].im);
        }
    }
}


// ------------------------------------------------- triangle-pair assembly
// The same quadrature sums as assemble_kernel, organised by triangle pairs:
// every RWG half on triangle a paired with every half on triangle b uses the
// same 7 x 7 Green's function values, so each (a, b) of a tile pair computes
// them once and keeps moments in coordinates relative to the centroids
// (u = r - c_a, v = r' - c_b, D = c_a - c_b, d = r - r' = D + u - v):
//   L: M0 = sum G, Mu = sum G u, Mv = sum G v, Muv = sum G u.v
//   K: S0 = sum g, A = sum g u, B = sum g v, C = sum g u x v, from which
//      (D being constant over the pair) P1 = sum g u.(D x v) = -D.C,
//      Q2 = sum g (u x D - u x v) = A x D - C, Q3 = sum g (D x v + u x v)
//      = D x B + C and Q4 = sum g d = D S0 + A - B
// (G, g with the weights jw jw').  With f_m = s_m (r - p_m) = s_m (u - pi_m),
// f_n = s_n (v - nu_n):
//   sum G f_m.f_n  = s_m s_n (Muv - pi.Mv - nu.Mu + pi.nu M0)
//   sum g f_m.(d x f_n) = s_m s_n (P1 - nu.Q2 - pi.Q3 + pi.(Q4 x nu))
// Each (RWG pair, half pair) term lands in its own shared-memory slot and the
// four half pairs of an entry are summed in a fixed order, so the result does
// not depend on the tiling.  RWGs are tiled in the Morton order of their
// triangles (geom_upload), ~17 distinct triangles per 16 RWGs: ~3.5x fewer
// Green's function evaluations than per RWG pair.
constexpr size_t tri_smem_bytes(int nmed) {
    return (size_t)2 * nmed * 1024 * sizeof(double2) +
           sizeof(double) * (2 * ASM_TRI_MAX * 3 + 2 * ASM_TRI_MAX * MAXQ * 3 + 2 * ASM_TRI_MAX * MAXQ +
                             2 * TILE * 2 * 5) +
           sizeof(int) * (2 * ASM_TRI_MAX + 2) + 2 * ASM_TRI_MAX * 3;
}

template <int NMED>
__global__ void __launch_bounds__(256, 2) assemble_tri_kernel(AsmArgs a, DevTriAsm ta) {
    int64_t lin = blockIdx.x;
    const int T = a.ntile;
    int bi = (int)floor((2.0 * T + 1.0 - sqrt((2.0 * T + 1.0) * (2.0 * T + 1.0) - 8.0 * (double)lin)) * 0.5);
    if (bi < 0) bi = 0;
    while (bi > 0 && (int64_t)bi * T - (int64_t)bi * (bi - 1) / 2 > lin) bi--;
    while ((int64_t)(bi + 1) * T - (int64_t)(bi + 1) * bi / 2 <= lin) bi++;
    const int bj = bi + (int)(lin - ((int64_t)bi * T - (int64_t)bi * (bi - 1) / 2));
    if (a.tile_flag && !a.tile_flag[bi] && !a.tile_flag[bj]) return;  // a tile the caller keeps
    const int N = a.N, Nq = a.Nq, tid = threadIdx.x;

    extern __shared__ __align__(16) unsigned char tri_smem[];
    double2* sL = reinterpret_cast<double2*>(tri_smem);  // [NMED][256 entries][4 half pairs]
    double2* sK = sL + NMED * 1024;
    double* sc = reinterpret_cast<double*>(sK + NMED * 1024);  // [2][TRI_MAX][3]
    double* su = sc + 2 * ASM_TRI_MAX * 3;                      // [2][TRI_MAX][MAXQ][3]
    double* sjw = su + 2 * ASM_TRI_MAX * MAXQ * 3;              // [2][TRI_MAX][MAXQ]
    double* ssig = sjw + 2 * ASM_TRI_MAX * MAXQ;                // [2][TILE][2]
    double* sdiv = ssig + 2 * TILE * 2;                         // [2][TILE][2]
    double* spi = sdiv + 2 * TILE * 2;                          // [2][TILE][2][3]
    int* stri = reinterpret_cast<int*>(spi + 2 * TILE * 2 * 3);  // [2][TRI_MAX]
    int* sntri = stri + 2 * ASM_TRI_MAX;                         // [2]
    unsigned char* sent = reinterpret_cast<unsigned char*>(sntri + 2);  // [2][TRI_MAX][3]

    for (int i = tid; i < 2 * ASM_TRI_MAX; i += blockDim.x) {
        const int side = i / ASM_TRI_MAX, li = i % ASM_TRI_MAX;
        const int t = ta.tile_tri[(size_t)(side ? bj : bi) * ASM_TRI_MAX + li];
        stri[i] = t;
        for (int j = 0; j < 3; j++) sc[i * 3 + j] = t >= 0 ? ta.c[(size_t)t * 3 + j] : 0.0;
    }
    for (int i = tid; i < 2 * ASM_TRI_MAX * Nq; i += blockDim.x) {
        const int q = i % Nq, sl = i / Nq;  // sl = side * TRI_MAX + li
        const int t = ta.tile_tri[(size_t)(sl >= ASM_TRI_MAX ? bj : bi) * ASM_TRI_MAX + sl % ASM_TRI_MAX];
        for (int j = 0; j < 3; j++) su[(sl * MAXQ + q) * 3 + j] = t >= 0 ? ta.u[((size_t)t * Nq + q) * 3 + j] : 0.0;
        sjw[sl * MAXQ + q] = t >= 0 ? ta.jw[(size_t)t * Nq + q] : 0.0;
    }
    for (int i = tid; i < 2 * ASM_TRI_MAX * 3; i += blockDim.x) {
        const int side = i / (ASM_TRI_MAX * 3);
        sent[i] = ta.tile_ent[(size_t)(side ? bj : bi) * ASM_TRI_MAX * 3 + i % (ASM_TRI_MAX * 3)];
    }
    for (int i = tid; i < 2 * TILE * 2; i += blockDim.x) {
        const int side = i / (TILE * 2), slot = (i / 2) % TILE, h = i % 2;
        const int n = ta.tile_rwg[(size_t)(side ? bj : bi) * TILE + slot];
        const int hn = h * N + (n >= 0 ? n : 0);
        ssig[i] = n >= 0 ? a.coef[hn] : 0.0;
        sdiv[i] = n >= 0 ? a.h.div[hn] : 0.0;
        for (int j = 0; j < 3; j++) spi[i * 3 + j] = n >= 0 ? ta.pi[(size_t)hn * 3 + j] : 0.0;
    }
    if (tid < 2) sntri[tid] = ta.tile_ntri[tid ? bj : bi];
    __syncthreads();

    const int na = sntri[0], nb = sntri[1];
    const bool exact = (a.flags & BEM_ASM_GSMOOTH_EXACT) != 0;
    const int items = na * nb * NMED;
    for (int it = tid; it < items; it += blockDim.x) {
        // medium-major: the lanes of a warp take the same branches (the
        // exterior medium is lossless, the interior one takes exp)
        const int e = it / (na * nb), pr = it % (na * nb), ia = pr / nb, ib = ASM_TRI_MAX + pr % nb;
        const bool same = stri[ia] == stri[ib];
        const Medium k = a.med[e];
        const double Dx = sc[ia * 3] - sc[ib * 3], Dy = sc[ia * 3 + 1] - sc[ib * 3 + 1],
                     Dz = sc[ia * 3 + 2] - sc[ib * 3 + 2];
        cplx M0 = {0, 0}, Muv = {0, 0}, S0 = {0, 0};
        cplx Mu[3], Mv[3], A[3], B[3], C[3];
#pragma unroll
        for (int j = 0; j < 3; j++) Mu[j] = Mv[j] = A[j] = B[j] = C[j] = {0, 0};
        for (int qa = 0; qa < Nq; qa++) {
            const double* up = &su[(ia * MAXQ + qa) * 3];
            const double ux = up[0], uy = up[1], uz = up[2], wa = sjw[ia * MAXQ + qa];
            for (int qb = 0; qb < Nq; qb++) {
                const double* vp = &su[(ib * MAXQ + qb) * 3];
                const double vx = vp[0], vy = vp[1], vz = vp[2], w = wa * sjw[ib * MAXQ + qb];
                const double dx = Dx + (ux - vx), dy = Dy + (uy - vy), dz = Dz + (uz - vz);
                // 1/R from one reciprocal square root (R clamped at 1e-15 as
                // R^2 at 1e-30); R = R^2 / R
                const double R2 = fmax(dx * dx + dy * dy + dz * dz, 1e-30);
                const double invR = rsqrt(R2), Rs = R2 * invR, R = Rs;
                const double i4R = __dmul_rn(INV4PI_D, invR);  // rounded alone, as in assemble_kernel
                double sn, cs;
                sincos(k.kr * Rs, &sn, &cs);
                const double ea = (k.ki != 0.0) ? exp_decay(k.ki * Rs) : 1.0;
                const cplx G = {ea * cs * i4R, ea * sn * i4R};
                cplx Gu = G;
                if (same) {
                    if (exact) Gu = g_smooth_exact(k, R);
                    else Gu.re -= i4R;
                }
                const cplx Gj = {Gu.re * w, Gu.im * w};
                const double uv = ux * vx + uy * vy + uz * vz;
                M0.re += Gj.re, M0.im += Gj.im;
                Muv.re += Gj.re * uv, Muv.im += Gj.im * uv;
                Mu[0].re += Gj.re * ux, Mu[0].im += Gj.im * ux;
                Mu[1].re += Gj.re * uy, Mu[1].im += Gj.im * uy;
                Mu[2].re += Gj.re * uz, Mu[2].im += Gj.im * uz;
                Mv[0].re += Gj.re * vx, Mv[0].im += Gj.im * vx;
                Mv[1].re += Gj.re * vy, Mv[1].im += Gj.im * vy;
                Mv[2].re += Gj.re * vz, Mv[2].im += Gj.im * vz;
                if (!same && R > 1e-12) {
                    const cplx gc = cmul(G, cplx{(-k.ki - invR) * invR, k.kr * invR});
                    const cplx gw = {gc.re * w, gc.im * w};
                    const double uu[3] = {ux, uy, uz}, vv[3] = {vx, vy, vz};
                    const double cr[3] = {uy * vz - uz * vy, uz * vx - ux * vz, ux * vy - uy * vx};
                    S0.re += gw.re, S0.im += gw.im;
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        A[j].re += gw.re * uu[j], A[j].im += gw.im * uu[j];
                        B[j].re += gw.re * vv[j], B[j].im += gw.im * vv[j];
                        C[j].re += gw.re * cr[j], C[j].im += gw.im * cr[j];
                    }
                }
            }
        }
        // P1 = -D.C, Q2 = A x D - C, Q3 = D x B + C, Q4 = D S0 + A - B
        const double DD[3] = {Dx, Dy, Dz};
        cplx P1 = {0, 0}, Q2[3], Q3[3], Q4[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            P1.re -= DD[j] * C[j].re, P1.im -= DD[j] * C[j].im;
            Q2[j] = {A[j1].re * DD[j2] - A[j2].re * DD[j1] - C[j].re, A[j1].im * DD[j2] - A[j2].im * DD[j1] - C[j].im};
            Q3[j] = {DD[j1] * B[j2].re - DD[j2] * B[j1].re + C[j].re, DD[j1] * B[j2].im - DD[j2] * B[j1].im + C[j].im};
            Q4[j] = {DD[j] * S0.re + A[j].re - B[j].re, DD[j] * S0.im + A[j].im - B[j].im};
        }
        const cplx ik = {-k.ki, k.kr};
        const double k2 = k.kr * k.kr + k.ki * k.ki;
        const cplx iok = {k.ki / k2, k.kr / k2};  // i/k
        for (int x = 0; x < 3; x++) {
            const int er = sent[ia * 3 + x];
            if (er == 0xff) break;
            const int r = er >> 1, hr = er & 1;
            const double sr = ssig[(r)*2 + hr], dr = sdiv[(r)*2 + hr];
            const double* pp = &spi[((r)*2 + hr) * 3];
            for (int y = 0; y < 3; y++) {
                const int ec = sent[ib * 3 + y];
                if (ec == 0xff) break;
                const int c = ec >> 1, hc = ec & 1;
                const double scn = ssig[(TILE + c) * 2 + hc], dc = sdiv[(TILE + c) * 2 + hc];
                const double* nn = &spi[((TILE + c) * 2 + hc) * 3];
                const double ss = sr * scn, pn = pp[0] * nn[0] + pp[1] * nn[1] + pp[2] * nn[2];
                cplx lv = {Muv.re + pn * M0.re, Muv.im + pn * M0.im};
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    lv.re -= pp[j] * Mv[j].re + nn[j] * Mu[j].re;
                    lv.im -= pp[j] * Mv[j].im + nn[j] * Mu[j].im;
                }
                lv.re *= ss, lv.im *= ss;
                const double dd = dr * dc;
                const cplx ls = {dd * M0.re, dd * M0.im};
                const cplx t1 = cmul(ik, lv), t2 = cmul(iok, ls);
                cplx kv = P1;
                // pi . (Q4 x nu)
                const cplx qx[3] = {{Q4[1].re * nn[2] - Q4[2].re * nn[1], Q4[1].im * nn[2] - Q4[2].im * nn[1]},
                                    {Q4[2].re * nn[0] - Q4[0].re * nn[2], Q4[2].im * nn[0] - Q4[0].im * nn[2]},
                                    {Q4[0].re * nn[1] - Q4[1].re * nn[0], Q4[0].im * nn[1] - Q4[1].im * nn[0]}};
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    kv.re += pp[j] * qx[j].re - nn[j] * Q2[j].re - pp[j] * Q3[j].re;
                    kv.im += pp[j] * qx[j].im - nn[j] * Q2[j].im - pp[j] * Q3[j].im;
                }
                const int slot = (r * TILE + c) * 4 + hr * 2 + hc;
                sL[e * 1024 + slot] = make_double2(t1.re - t2.re, t1.im - t2.im);
                sK[e * 1024 + slot] = make_double2(ss * kv.re, ss * kv.im);
            }
        }
    }
    __syncthreads();

    const int r = tid / TILE, c = tid % TILE;
    const int mm = ta.tile_rwg[(size_t)bi * TILE + r], n = ta.tile_rwg[(size_t)bj * TILE + c];
    if (mm < 0 || n < 0) return;
    if (bi == bj && c < r) return;  // diagonal tile pair: the upper entry writes both positions
    cplx Lf[NMED], Kk[NMED];
#pragma unroll
    for (int e = 0; e < NMED; e++) {
        const double2* l = &sL[e * 1024 + (r * TILE + c) * 4];
        const double2* kk = &sK[e * 1024 + (r * TILE + c) * 4];
        Lf[e] = {((l[0].x + l[1].x) + l[2].x) + l[3].x, ((l[0].y + l[1].y) + l[2].y) + l[3].y};
        Kk[e] = {((kk[0].x + kk[1].x) + kk[2].x) + kk[3].x, ((kk[0].y + kk[1].y) + kk[2].y) + kk[3].y};
    }
    const bool mirror = (n != mm);
    if (a.Z) {
        cplx TL, BR, Ks;
        if constexpr (NMED == 2) {
            TL = {a.eta_e * Lf[0].re + a.eta_i * Lf[1].re, a.eta_e * Lf[0].im + a.eta_i * Lf[1].im};
            BR = {Lf[0].re / a.eta_e + Lf[1].re / a.eta_i, Lf[0].im / a.eta_e + Lf[1].im / a.eta_i};
            Ks = {Kk[0].re + Kk[1].re, Kk[0].im + Kk[1].im};
        } else {
            TL = {a.eta_e * Lf[0].re, a.eta_e * Lf[0].im};
            BR = {Lf[0].re / a.eta_e, Lf[0].im / a.eta_e};
            Ks = Kk[0];
        }
        double2* Z = a.Z;
        const int64_t ld = a.ldz;
        Z[(int64_t)mm * ld + n] = make_double2(TL.re, TL.im);
        Z[(int64_t)mm * ld + N + n] = make_double2(-Ks.re, -Ks.im);
        Z[(int64_t)(N + mm) * ld + n] = make_double2(Ks.re, Ks.im);
        Z[(int64_t)(N + mm) * ld + N + n] = make_double2(BR.re, BR.im);
        if (mirror) {
            Z[(int64_t)n * ld + mm] = make_double2(TL.re, TL.im);
            Z[(int64_t)n * ld + N + mm] = make_double2(-Ks.re, -Ks.im);
            Z[(int64_t)(N + n) * ld + mm] = make_double2(Ks.re, Ks.im);
            Z[(int64_t)(N + n) * ld + N + mm] = make_double2(BR.re, BR.im);
        }
    } else {
        a.L[(int64_t)mm * a.ld + n] = make_double2(Lf[0].re, Lf[0].im);
        a.K[(int64_t)mm * a.ld + n] = make_double2(Kk[0].re, Kk[0].im);
        if (mirror) {
            a.L[(int64_t)n * a.ld + mm] = make_double2(Lf[0].re, Lf[0].im);
            a.K[(int64_t)n * a.ld + mm] = make_double2(Kk[0].re, Kk[0].im);
        }
    }
}

// Tiles to recompute from an RWG mask (tile_rwg null: tiles of 16
// consecutive RWGs), and per RWG whether its tile is recomputed.
__global__ void mask_tiles_kernel(const unsigned char* __restrict__ mask, const int* __restrict__ tile_rwg, int N,
                                  int ntile, unsigned char* __restrict__ flag) {
    const int tl = blockIdx.x * blockDim.x + threadIdx.x;
    if (tl >= ntile) return;
    unsigned char f = 0;
    for (int sl = 0; sl < TILE; sl++) {
        const int n = tile_rwg ? tile_rwg[(size_t)tl * TILE + sl] : tl * TILE + sl;
        if (n >= 0 && n < N && mask[n]) f = 1;
    }
    flag[tl] = f;
}

__global__ void mask_rec_kernel(const unsigned char* __restrict__ flag, const int* __restrict__ pos, int N,
                                unsigned char* __restrict__ rec) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    rec[n] = flag[(pos ? pos[n] : n) / TILE];
}

// ------------------------------------------------------------ singular fixup
struct FixArgs {
    DevHalf h;
    DevSingular s;
    const double* coef;  // (2N) sign*l/(2A)
    const double* fr;    // (3*2N) free vertex: x block, y block, z block
    int N, Nq, nmed;
    Medium med[2];
    double eta_e, eta_i;
    double2* Z;
    int64_t ldz;
    double2* L;
    int64_t ld;
    const unsigned char* rec;   // optional: RWGs whose assembly tiles were recomputed
};

// One thread per unordered RWG pair {m, n} sharing a triangle.  For every
// (triangle t, test half a, source half b) item:
//   A = div_a div_b sum_q P_q jw_a,q / (4 pi)
//   B = sum_q f_a,q . coef_b (V_q - r_free,b P_q) jw_a,q / (4 pi)
// and S = -(i/k) A + i k B (assembly.cu:290-317).  The symmetrised
// correction (S[m,n] + S[n,m])/2 is added to both L entries.
__global__ void singular_fixup_kernel(FixArgs a) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.s.npairs) return;
    const int N = a.N, Nq = a.Nq;
    int m = a.s.pair_mn[2 * p], n = a.s.pair_mn[2 * p + 1];
    if (a.rec && !a.rec[m] && !a.rec[n]) return;
    double SA = 0.0, SB = 0.0;
    for (int it = a.s.item_ptr[p]; it < a.s.item_ptr[p + 1]; it++) {
        int t = a.s.item[3 * it], ha = a.s.item[3 * it + 1], hb = a.s.item[3 * it + 2];
        double sbase = 0.0, vec = 0.0;
        double cb = a.coef[hb];
        double frx = a.fr[hb], fry = a.fr[2 * N + hb], frz = a.fr[4 * N + hb];
        for (int q = 0; q < Nq; q++) {
            size_t ip = (size_t)ha * Nq + q;
            size_t tq = (size_t)t * Nq + q;
            double P = a.s.P[tq];
            double jw = a.h.jw[ip];
            sbase += P * jw;
            double gx = cb * (a.s.V[3 * tq] - frx * P);
            double gy = cb * (a.s.V[3 * tq + 1] - fry * P);
            double gz = cb * (a.s.V[3 * tq + 2] - frz * P);
            vec += (a.h.fx[ip] * gx + a.h.fy[ip] * gy + a.h.fz[ip] * gz) * jw;
        }
        SA += a.h.div[ha] * a.h.div[hb] * (sbase * INV4PI_D);
        SB += vec * INV4PI_D;
    }
    if (m != n) {
        SA *= 0.5;
        SB *= 0.5;
    }
    cplx dL[2];
    for (int e = 0; e < a.nmed; e++) {
        Medium k = a.med[e];
        double k2 = k.kr * k.kr + k.ki * k.ki;
        cplx iok = {k.ki / k2, k.kr / k2};
        cplx ik = {-k.ki, k.kr};
        dL[e] = {-iok.re * SA + ik.re * SB, -iok.im * SA + ik.im * SB};
    }
    if (a.Z) {
        cplx TL, BR;
        if (a.nmed == 2) {
            TL = {a.eta_e * dL[0].re + a.eta_i * dL[1].re, a.eta_e * dL[0].im + a.eta_i * dL[1].im};
            BR = {dL[0].re / a.eta_e + dL[1].re / a.eta_i, dL[0].im / a.eta_e + dL[1].im / a.eta_i};
        } else {
            TL = {a.eta_e * dL[0].re, a.eta_e * dL[0].im};
            BR = {dL[0].re / a.eta_e, dL[0].im / a.eta_e};
        }
        double2* z;
        z = &a.Z[(int64_t)m * a.ldz + n];
        z->x += TL.re, z->y += TL.im;
        z = &a.Z[(int64_t)(N + m) * a.ldz + N + n];
        z->x += BR.re, z->y += BR.im;
        if (m != n) {
            z = &a.Z[(int64_t)n * a.ldz + m];
            z->x += TL.re, z->y += TL.im;
            z = &a.Z[(int64_t)(N + n) * a.ldz + N + m];
            z->x += BR.re, z->y += BR.im;
        }
    } else {
        double2* z = &a.L[(int64_t)m * a.ld + n];
        z->x += dL[0].re, z->y += dL[0].im;
        if (m != n) {
            z = &a.L[(int64_t)n * a.ld + m];
            z->x += dL[0].re, z->y += dL[0].im;
        }
    }
}

// mode 2: PMCHWT into Z; mode 1: L and K of medium 0 into L, K; mode 3: the
// exterior-only PMCHWT A_ext of medium 0 into Z.
int assemble_dev(bem_ctx* ctx, const bem_geom* g, double ke_re, double ke_im, double ki_re,
                 double ki_im, double eta_e, double eta_i, unsigned flags, int mode, void* Z,
                 int64_t ldz, void* L, void* K, const unsigned char* rwg_mask) {
    const int N = g->N;
    if (N < 1) return fail(ctx, BEM_ERR_INVALID, "empty basis");
    if ((mode == 2 || mode == 3) && (!Z || ldz < 2 * N)) return fail(ctx, BEM_ERR_INVALID, "bad Z / ldz");
    if (mode == 1 && (!L || !K || ldz < N)) return fail(ctx, BEM_ERR_INVALID, "bad L/K / ld");
    if (!(ke_re != 0.0 || ke_im != 0.0) || (mode == 2 && !(ki_re != 0.0 || ki_im != 0.0)))
        return fail(ctx, BEM_ERR_INVALID, "zero wavenumber");
    if (mode == 2 && (!(eta_e > 0) || !(eta_i > 0))) return fail(ctx, BEM_ERR_INVALID, "eta <= 0");
    if (mode == 3 && !(eta_e > 0)) return fail(ctx, BEM_ERR_INVALID, "eta <= 0");
    const int nmed = mode == 2 ? 2 : 1;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    // 1. Graglia P, V per (triangle, point)
    TriQ tq;
    tq.n = g->quad.n;
    for (int i = 0; i < 25; i++) tq.l1[i] = g->quad.l1[i], tq.l2[i] = g->quad.l2[i], tq.w[i] = g->quad.w[i];
    int nthr = g->nt * g->Nq;
    graglia_kernel<<<(nthr + 127) / 128, 128, 0, st>>>(g->sing.tv, g->nt, tq, g->sing.P, g->sing.V);
    BEM_LAUNCHED(ctx);
    // 2. quadrature part, upper tiles
    AsmArgs a;
    a.h = g->half;
    a.N = N;
    a.Nq = g->Nq;
    a.ntile = (N + TILE - 1) / TILE;
    a.med[0] = {ke_re, ke_im};
    a.med[1] = {ki_re, ki_im};
    a.eta_e = eta_e;
    a.eta_i = eta_i;
    a.flags = flags;
    a.Z = mode == 1 ? nullptr : (double2*)Z;
    a.ldz = ldz;
    a.L = (double2*)L;
    a.K = (double2*)K;
    a.ld = ldz;
    a.coef = g->sing_coef;
    a.tile_flag = nullptr;
    const bool tri = ctx->asm_kernel == 0;
    const unsigned char* rec = nullptr;
    if (rwg_mask) {
        // tiles holding a flagged RWG, and the RWGs of those tiles
        mask_tiles_kernel<<<(a.ntile + 127) / 128, 128, 0, st>>>(rwg_mask, tri ? g->tri.tile_rwg : nullptr, N,
                                                                 a.ntile, g->tri.tile_flag);
        BEM_LAUNCHED(ctx);
        mask_rec_kernel<<<(N + 255) / 256, 256, 0, st>>>(g->tri.tile_flag, tri ? g->tri.pos : nullptr, N,
                                                         g->tri.rwg_rec);
        BEM_LAUNCHED(ctx);
        a.tile_flag = g->tri.tile_flag;
        rec = g->tri.rwg_rec;
    }
    int64_t ntiles = (int64_t)a.ntile * (a.ntile + 1) / 2;
    if (ntiles > 0x7fffffffLL) return fail(ctx, BEM_ERR_INVALID, "too many tiles");
    if (g->Nq > MAXQ) return fail(ctx, BEM_ERR_INVALID, "quadrature of %d points (at most %d)", g->Nq, MAXQ);
    cudaEvent_t ev = ctx->prof_begin(PROF_ASSEMBLY);
    if (tri) {
        // dynamic shared memory beyond 48 KB: set once per device
        static unsigned attr_done = 0;
        const unsigned bit = 1u << (ctx->device & 31);
        if (!(__atomic_load_n(&attr_done, __ATOMIC_ACQUIRE) & bit)) {
            BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(assemble_tri_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)tri_smem_bytes(2)));
            BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(assemble_tri_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)tri_smem_bytes(1)));
            __atomic_fetch_or(&attr_done, bit, __ATOMIC_RELEASE);
        }
        if (mode == 2)
            assemble_tri_kernel<2><<<(unsigned)ntiles, 256, tri_smem_bytes(2), st>>>(a, g->tri);
        else
            assemble_tri_kernel<1><<<(unsigned)ntiles, 256, tri_smem_bytes(1), st>>>(a, g->tri);
    } else if (mode == 2) {
        assemble_kernel<2><<<(unsigned)ntiles, 256, 0, st>>>(a);
    } else {
        assemble_kernel<1><<<(unsigned)ntiles, 256, 0, st>>>(a);
    }
    BEM_LAUNCHED(ctx);
    // algorithmic unit: one quadrature-pair evaluation per medium, every
    // ordered RWG pair (no symmetry credit): 64 flop + sincos + exp each
    if (ev)
        ctx->prof_end(PROF_ASSEMBLY, ev, 64.0 * nmed * 4.0 * N * (double)N * g->Nq * g->Nq,
                      (mode == 1 ? 32.0 : 64.0) * (double)N * N);
    // 3. singular correction
    if (g->sing.npairs > 0) {
        FixArgs f;
        f.h = g->half;
        f.s = g->sing;
        f.coef = g->sing_coef;
        f.fr = g->sing_free;
        f.N = N;
        f.Nq = g->Nq;
        f.nmed = nmed;
        f.med[0] = {ke_re, ke_im};
        f.med[1] = {ki_re, ki_im};
        f.eta_e = eta_e;
        f.eta_i = eta_i;
        f.Z = a.Z;
        f.ldz = ldz;
        f.L = (double2*)L;
        f.ld = ldz;
        f.rec = rec;
        singular_fixup_kernel<<<(g->sing.npairs + 127) / 128, 128, 0, st>>>(f);
        BEM_LAUNCHED(ctx);
    }
    return BEM_OK;
}

}  // namespace bem

using namespace bem;

extern "C" {

int bem_geom_create(bem_ctx* ctx, const double* verts, int nv, const int* tris, int nt,
                    int quad_order, bem_geom** out, int* N) {
    if (!ctx || !out) return BEM_ERR_INVALID;
    *out = nullptr;
    bem_geom* g = new bem_geom();
    g->ctx = ctx;
    g->device = ctx->device;
    if (!host_mesh_from(verts, nv, tris, nt, &g->mesh)) {
        delete g;
        return fail(ctx, BEM_ERR_INVALID, "bad mesh arrays");
    }
    if (!quadrature(quad_order, &g->quad)) {
        delete g;
        return fail(ctx, BEM_ERR_INVALID, "quadrature order %d unsupported (4, 7, 13)", quad_order);
    }
    g->quad_order = quad_order;
    g->rwg = build_rwg(g->mesh);
    g->N = g->rwg.N;
    g->Nq = g->quad.n;
    g->nv = nv;
    g->nt = nt;
    if (g->N < 1) {
        delete g;
        return fail(ctx, BEM_ERR_INVALID, "mesh has no interior edges");
    }
    int s = cudaSetDevice(ctx->device) == cudaSuccess ? geom_upload(ctx, g) : BEM_ERR_CUDA;
    if (s != BEM_OK) {
        if (g->dmem) devmem_free(ctx->device, g->dmem, g->dmem_bytes, ctx);
        delete g;
        return s;
    }
    *out = g;
    if (N) *N = g->N;
    return BEM_OK;
}

int bem_geom_create_rwg(bem_ctx* ctx, const double* verts, int nv, const int* tris, int nt, int N,
                        const int* tri_p, const int* tri_m, const double* free_p, const double* free_m,
                        const double* length, const double* area_p, const double* area_m, int quad_order,
                        bem_geom** out) {
    if (!ctx || !out || N < 1 || !tri_p || !tri_m || !free_p || !free_m || !length || !area_p || !area_m)
        return BEM_ERR_INVALID;
    *out = nullptr;
    bem_geom* g = new bem_geom();
    g->ctx = ctx;
    g->device = ctx->device;
    if (!host_mesh_from(verts, nv, tris, nt, &g->mesh) || !quadrature(quad_order, &g->quad)) {
        delete g;
        return fail(ctx, BEM_ERR_INVALID, "bad mesh arrays or quadrature order");
    }
    HostRWG& r = g->rwg;
    r.N = N;
    for (int n = 0; n < N; n++) {
        if (tri_p[n] < 0 || tri_p[n] >= nt || tri_m[n] < 0 || tri_m[n] >= nt) {
            delete g;
            return fail(ctx, BEM_ERR_INVALID, "RWG %d refers to a missing triangle", n);
        }
        r.tri_p.push_back(tri_p[n]);
        r.tri_m.push_back(tri_m[n]);
        r.vfree_p.push_back(-1);
        r.vfree_m.push_back(-1);
        r.free_p.push_back({free_p[3 * n], free_p[3 * n + 1], free_p[3 * n + 2]});
        r.free_m.push_back({free_m[3 * n], free_m[3 * n + 1], free_m[3 * n + 2]});
        r.length.push_back(length[n]);
        r.area_p.push_back(area_p[n]);
        r.area_m.push_back(area_m[n]);
    }
    g->quad_order = quad_order;
    g->N = N;
    g->Nq = g->quad.n;
    g->nv = nv;
    g->nt = nt;
    int s = cudaSetDevice(ctx->device) == cudaSuccess ? geom_upload(ctx, g) : BEM_ERR_CUDA;
    if (s != BEM_OK) {
        if (g->dmem) devmem_free(ctx->device, g->dmem, g->dmem_bytes, ctx);
        delete g;
        return s;
    }
    *out = g;
    return BEM_OK;
}

int bem_geom_free(bem_geom* g) {
    if (!g) return BEM_OK;
    if (g->dmem) {
        cudaSetDevice(g->device);
        // last used on the creating context's stream (or the device waits)
        devmem_free(g->device, g->dmem, g->dmem_bytes, g->ctx);
    }
    delete g;
    return BEM_OK;
}

int bem_geom_size(const bem_geom* g) { return g ? g->N : 0; }

int bem_geom_set_vertices(bem_ctx* ctx, bem_geom* g, const double* verts) {
    if (!ctx || !g || !verts) return BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    return geom_set_vertices(ctx, g, verts);
}

int bem_assemble_pmchwt_dev(bem_ctx* ctx, const bem_geom* g, double kext_re, double kext_im,
                            double kint_re, double kint_im, double eta_ext, double eta_int,
                            unsigned flags, void* Z_dev, int64_t ldz) {
    if (!ctx || !g) return BEM_ERR_INVALID;
    return assemble_dev(ctx, g, kext_re, kext_im, kint_re, kint_im, eta_ext, eta_int, flags, 2,
                        Z_dev, ldz, nullptr, nullptr);
}

int bem_assemble_aext_dev(bem_ctx* ctx, const bem_geom* g, double kext_re, double kext_im, double eta_ext,
                          unsigned flags, void* Z_dev, int64_t ldz) {
    if (!ctx || !g) return BEM_ERR_INVALID;
    return assemble_dev(ctx, g, kext_re, kext_im, 0, 0, eta_ext, 1, flags, 3, Z_dev, ldz, nullptr, nullptr);
}

int bem_assemble_LK_dev(bem_ctx* ctx, const bem_geom* g, double k_re, double k_im,
                        unsigned flags, void* L_dev, void* K_dev, int64_t ld) {
    if (!ctx || !g) return BEM_ERR_INVALID;
    return assemble_dev(ctx, g, k_re, k_im, 0, 0, 1, 1, flags, 1, nullptr, ld, L_dev, K_dev);
}

}  // extern "C"
