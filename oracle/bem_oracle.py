"""CPU oracle for the dense PMCHWT path (TEST INFRASTRUCTURE ONLY).

This module is a plain NumPy/SciPy restatement of the reference's FP64 dense
path.  It exists to check the CUDA implementation; nothing in the product
imports it.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may use it.

Every function cites the reference file and lines it restates (paths relative
to the KirillSalnikov/BEM-CPP project root).  The oracle is pinned against
golden vectors produced by running the reference's own ``python/bem_core.py``
(see ``tests/golden/make_golden.py``) and, for hexagonal prisms, the
reference's own C++ mesher compiled by ``oracle/Makefile``.

Third-party arithmetic: the dense LU and the triangular solves go through
LAPACK ``zgetrf``/``zgetrs`` via ``scipy.linalg.lu_factor``/``lu_solve``,
exactly the calls the reference's CPU path makes (bem_core.py:1637, 1713).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

INV4PI = 1.0 / (4.0 * math.pi)


# ---------------------------------------------------------------------------
# a1. Meshes
# ---------------------------------------------------------------------------

_ICO_TRIS = np.array([
    [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
    [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
    [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
    [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
], dtype=np.int64)


def _midpoint_subdivide(verts, tris, project):
    """One 1->4 midpoint split; new vertex per edge in first-visit order.

    Restates mesh.cpp:27-56 (icosphere loop) and mesh.cpp:70-100
    (subdivide_flat): child triangles (a,ab,ca), (b,bc,ab), (c,ca,bc), (ab,bc,ca).
    """
    verts = [np.asarray(v, dtype=np.float64) for v in verts]
    mid = {}

    def get_mid(a, b):
        key = (min(a, b), max(a, b))
        if key in mid:
            return mid[key]
        m = (verts[a] + verts[b]) * 0.5
        if project:
            m = m / math.sqrt(float(m @ m))
        verts.append(m)
        mid[key] = len(verts) - 1
        return mid[key]

    out = []
    for a, b, c in tris:
        a, b, c = int(a), int(b), int(c)
        ab = get_mid(a, b)
        bc = get_mid(b, c)
        ca = get_mid(c, a)
        out += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
    return np.array(verts), np.array(out, dtype=np.int64)


def icosphere(radius=1.0, refinements=2):
    """Icosphere by midpoint subdivision with projection (mesh.cpp:11-68,
    bem_core.py:24-61)."""
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([
        [-1, phi, 0], [1, phi, 0], [-1, -phi, 0], [1, -phi, 0],
        [0, -1, phi], [0, 1, phi], [0, -1, -phi], [0, 1, -phi],
        [phi, 0, -1], [phi, 0, 1], [-phi, 0, -1], [-phi, 0, 1],
    ], dtype=np.float64)
    v = v * (1.0 / math.sqrt(float(v[0] @ v[0])))
    t = _ICO_TRIS.copy()
    for _ in range(refinements):
        v, t = _midpoint_subdivide(v, t, project=True)
    return v * radius, t


def subdivide_flat(verts, tris):
    """Flat midpoint subdivision (mesh.cpp:70-100)."""
    return _midpoint_subdivide(verts, tris, project=False)


def hex_prism(aspect_ratio, refinements):
    """Hexagonal prism of unit equivalent-sphere radius (mesh.cpp:102-154).

    a = (8*pi/(27*AR))^(1/3), H = AR*a*sqrt(3); 14 vertices, 24 triangles,
    then ``refinements`` flat subdivisions.
    """
    a = (8.0 * math.pi / (27.0 * aspect_ratio)) ** (1.0 / 3.0)
    H = aspect_ratio * a * math.sqrt(3.0)
    v = np.zeros((14, 3))
    v[0] = (0, 0, H / 2)
    v[7] = (0, 0, -H / 2)
    for i in range(6):
        ang = 2.0 * math.pi * i / 6.0
        x, y = a * math.cos(ang), a * math.sin(ang)
        v[1 + i] = (x, y, H / 2)
        v[8 + i] = (x, y, -H / 2)
    t = []
    for i in range(6):
        i1, i2 = 1 + i, 1 + (i + 1) % 6
        j1, j2 = 8 + i, 8 + (i + 1) % 6
        t += [[0, i1, i2], [7, j2, j1], [i1, j1, j2], [i1, j2, i2]]
    t = np.array(t, dtype=np.int64)
    for _ in range(refinements):
        v, t = subdivide_flat(v, t)
    return v, t


def mesh_volume(verts, tris):
    """Signed volume of a closed mesh (mesh.cpp:252-261)."""
    v0, v1, v2 = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    return float(np.sum(np.einsum('ij,ij->i', v0, np.cross(v1, v2)))) / 6.0


# ---------------------------------------------------------------------------
# a2. RWG basis
# ---------------------------------------------------------------------------

def build_rwg(verts, tris, order="cpp"):
    """Interior edges shared by exactly two triangles -> RWG functions.

    ``order="cpp"`` sorts edges by (min vertex, max vertex) like the C++
    std::map (rwg.cpp:5-43); ``order="python"`` keeps first-visit order like
    the Python dict (bem_core.py:397-421).  In both, the first triangle that
    visits the edge is the plus triangle and its opposite vertex is free_p.
    """
    edges = {}
    for ti, tri in enumerate(tris):
        for j in range(3):
            a, b, opp = int(tri[j]), int(tri[(j + 1) % 3]), int(tri[(j + 2) % 3])
            edges.setdefault((min(a, b), max(a, b)), []).append((ti, opp))
    keys = sorted(edges) if order == "cpp" else list(edges)
    tp, tm, fp, fm, ln = [], [], [], [], []
    for key in keys:
        lst = edges[key]
        if len(lst) != 2:
            continue
        (t_p, v_p), (t_m, v_m) = lst
        tp.append(t_p)
        tm.append(t_m)
        fp.append(v_p)
        fm.append(v_m)
        d = verts[key[1]] - verts[key[0]]
        ln.append(math.sqrt(float(d @ d)))
    tp = np.array(tp, dtype=np.int64)
    tm = np.array(tm, dtype=np.int64)
    area = tri_areas(verts, tris)
    return {
        "N": len(tp), "tri_p": tp, "tri_m": tm,
        "free_p": verts[np.array(fp, dtype=np.int64)],
        "free_m": verts[np.array(fm, dtype=np.int64)],
        "free_p_idx": np.array(fp, dtype=np.int64),
        "free_m_idx": np.array(fm, dtype=np.int64),
        "length": np.array(ln), "area_p": area[tp], "area_m": area[tm],
    }


def tri_areas(verts, tris):
    v0, v1, v2 = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    return 0.5 * np.linalg.norm(np.cross(v1 - v0, v2 - v0), axis=1)


# ---------------------------------------------------------------------------
# a3. Triangle quadrature (Dunavant)
# ---------------------------------------------------------------------------

def tri_quadrature(order=7):
    """Dunavant rules, barycentric (l1, l2), weights summing to 1
    (quadrature.h:14-70; bem_core.py:428-510).  Unknown orders fall back to 7
    like the C++ default branch."""
    if order == 4:
        pts = [[1 / 3, 1 / 3], [0.6, 0.2], [0.2, 0.6], [0.2, 0.2]]
        wts = [-27 / 48, 25 / 48, 25 / 48, 25 / 48]
    elif order == 13:
        a, b = 0.260345966079038, 0.479308067841923
        c, d = 0.065130102902216, 0.869739794195568
        e, f, g = 0.048690315425316, 0.312865496004875, 0.638444188569809
        pts = [[1 / 3, 1 / 3], [a, a], [a, b], [b, a], [c, c], [c, d], [d, c],
               [e, f], [f, e], [g, f], [f, g], [e, g], [g, e]]
        wa, wb, wc = 0.175615257433204, 0.053347235608839, 0.077113760890257
        wts = [-0.149570044467670] + [wa] * 3 + [wb] * 3 + [wc] * 6
    else:
        a1, a2 = 0.059715871789770, 0.470142064105115
        b1, b2 = 0.797426985353087, 0.101286507323456
        pts = [[1 / 3, 1 / 3], [a1, a2], [a2, a1], [a2, a2], [b1, b2], [b2, b1], [b2, b2]]
        w2, w3 = 0.13239415278851, 0.12593918054483
        wts = [0.225, w2, w2, w2, w3, w3, w3]
    return np.array(pts, dtype=np.float64), np.array(wts, dtype=np.float64)


def quad_points(verts, tris, tri_idx, pts):
    """Physical quadrature points r = l0 v0 + l1 v1 + l2 v2, shape (n, Nq, 3)."""
    t = tris[tri_idx]
    v0, v1, v2 = verts[t[:, 0]], verts[t[:, 1]], verts[t[:, 2]]
    lam0 = 1.0 - pts[:, 0] - pts[:, 1]
    return (lam0[None, :, None] * v0[:, None, :] + pts[None, :, 0, None] * v1[:, None, :]
            + pts[None, :, 1, None] * v2[:, None, :])


@dataclass
class Half:
    """Per-(RWG, half) quadrature data (assembly.cu:150-201, bem_core.py:807-829)."""
    qp: np.ndarray    # (N, Nq, 3)
    f: np.ndarray     # (N, Nq, 3)  sign*(l/2A)(r - r_free)
    div: np.ndarray   # (N,)        sign*l/A
    jw: np.ndarray    # (N, Nq)     A*w_q
    tri: np.ndarray   # (N,)
    sign: int
    free: np.ndarray  # (N, 3)
    coeff: np.ndarray  # (N,) l/(2A)  (unsigned)


def halves(rwg, verts, tris, quad_order=7):
    pts, wts = tri_quadrature(quad_order)
    out = []
    for sign, tri, free, area in ((+1, rwg["tri_p"], rwg["free_p"], rwg["area_p"]),
                                  (-1, rwg["tri_m"], rwg["free_m"], rwg["area_m"])):
        qp = quad_points(verts, tris, tri, pts)
        coeff = rwg["length"] / (2.0 * area)
        f = sign * coeff[:, None, None] * (qp - free[:, None, :])
        out.append(Half(qp=qp, f=f, div=sign * rwg["length"] / area,
                        jw=area[:, None] * wts[None, :], tri=tri, sign=sign,
                        free=free, coeff=coeff))
    return out


# ---------------------------------------------------------------------------
# a6. Graglia singular integrals (vectorised over observation points)
# ---------------------------------------------------------------------------

def potential_integral(r, v0, v1, v2):
    """int_T 1/|r - r'| dS' (Graglia 1993), vectorised over leading axes.

    Restates graglia.h:11-66 / bem_core.py:517-585 including its guards
    (edge length < 1e-15 skipped, log only when both R+s > 1e-15 and the
    ratio is positive, arctan only when |h| > 1e-15)."""
    r = np.asarray(r, dtype=np.float64)
    vs = (v0, v1, v2)
    n = np.cross(v1 - v0, v2 - v0)
    nn = np.linalg.norm(n, axis=-1, keepdims=True)
    nh = n / np.where(nn < 1e-15, 1.0, nn)
    res = np.zeros(r.shape[:-1])
    for i in range(3):
        vi, vj = vs[i], vs[(i + 1) % 3]
        e = vj - vi
        le = np.linalg.norm(e, axis=-1, keepdims=True)
        th = e / np.where(le < 1e-15, 1.0, le)
        mh = np.cross(nh, th)
        di = r - vi
        d = np.sum(di * mh, axis=-1)
        h = np.sum(di * nh, axis=-1)
        dj = vj - r
        dii = vi - r
        sp = np.sum(dj * th, axis=-1)
        sm = np.sum(dii * th, axis=-1)
        Rp = np.linalg.norm(dj, axis=-1)
        Rm = np.linalg.norm(dii, axis=-1)
        ok = (Rp + sp > 1e-15) & (Rm + sm > 1e-15)
        num = np.where(ok, Rp + sp, 1.0)
        den = np.where(ok, Rm + sm, 1.0)
        arg = num / den
        ok = ok & (arg > 0)
        term = np.where(ok, d * np.log(np.where(ok, arg, 1.0)), 0.0)
        ah = np.abs(h)
        R0sq = d * d + h * h
        t1 = np.arctan2(d * sp, R0sq + ah * Rp)
        t2 = np.arctan2(d * sm, R0sq + ah * Rm)
        term = term - np.where(ah > 1e-15, ah * (t1 - t2), 0.0)
        res = res + np.where(le[..., 0] < 1e-15, 0.0, term)
    return np.where(nn[..., 0] < 1e-15, 0.0, res)


def integral_R(r, v0, v1, v2, pts, wts):
    """int_T |r - r'| dS' by the triangle rule (graglia.h:69-85)."""
    lam0 = 1.0 - pts[:, 0] - pts[:, 1]
    q = (lam0[:, None] * v0[..., None, :] + pts[:, 0, None] * v1[..., None, :]
         + pts[:, 1, None] * v2[..., None, :])
    R = np.linalg.norm(q - r[..., None, :], axis=-1)
    area = 0.5 * np.linalg.norm(np.cross(v1 - v0, v2 - v0), axis=-1)
    return area * np.sum(wts * R, axis=-1)


def vector_potential_integral(r, v0, v1, v2, pts, wts, eps=1e-6):
    """int_T r'/|r - r'| dS' = r P - grad W with grad W by central differences
    of step eps=1e-6 (graglia.h:90-112, bem_core.py:705-715)."""
    P = potential_integral(r, v0, v1, v2)
    g = np.zeros(r.shape)
    for d in range(3):
        rp = r.copy()
        rm = r.copy()
        rp[..., d] += eps
        rm[..., d] -= eps
        g[..., d] = (integral_R(rp, v0, v1, v2, pts, wts)
                     - integral_R(rm, v0, v1, v2, pts, wts)) / (2.0 * eps)
    return P, r * P[..., None] - g


def singular_corrections(rwg, verts, tris, k, quad_order=7):
    """Same-triangle correction S (N x N, complex) to add to L before
    symmetrisation (assembly.cu:208-321, bem_core.py:718-780).

    S[m,n] += -(i/k) div_t div_s sum_q P_q jw_t,q / (4 pi)
              + i k sum_q f_t,q . s_sign s_coeff (V_q - r_free,s P_q) jw_t,q / (4 pi)
    over every (test half of m, source half of n) on the same triangle."""
    pts, wts = tri_quadrature(quad_order)
    N = rwg["N"]
    nt = len(tris)
    v0, v1, v2 = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    qp = quad_points(verts, tris, np.arange(nt), pts)          # (nt, Nq, 3)
    bc = lambda a: np.broadcast_to(a[:, None, :], qp.shape)
    P, V = vector_potential_integral(qp, bc(v0), bc(v1), bc(v2), pts, wts)
    H = halves(rwg, verts, tris, quad_order)
    ik = 1j * k
    ik_inv = 1j / k
    S = np.zeros((N, N), dtype=complex)
    # entries per triangle: (rwg index, half)
    per_tri = [[] for _ in range(nt)]
    for h_i, h in enumerate(H):
        for n in range(N):
            per_tri[int(h.tri[n])].append((n, h_i))
    for t in range(nt):
        ent = per_tri[t]
        if not ent:
            continue
        Pt, Vt = P[t], V[t]
        for (m, th) in ent:
            ht = H[th]
            tf, tjw, tdiv = ht.f[m], ht.jw[m], ht.div[m]
            scalar_base = float(np.dot(Pt, tjw)) * INV4PI
            for (n, sh) in ent:
                hs = H[sh]
                fn = hs.sign * hs.coeff[n] * (Vt - hs.free[n][None, :] * Pt[:, None])
                vec = float(np.sum(np.sum(tf * fn, axis=1) * tjw)) * INV4PI
                S[m, n] += -ik_inv * tdiv * hs.div[n] * scalar_base + ik * vec
    return S


# ---------------------------------------------------------------------------
# a5/a7. L and K operators, a8. PMCHWT system
# ---------------------------------------------------------------------------

def g_smooth(k, R):
    """(exp(ikR) - 1)/(4 pi R) without cancellation, limit ik/(4 pi) at R=0.

    With k = b + i c:  exp(ikR) - 1 = expm1(-cR) cos(bR) - 2 sin^2(bR/2)
    + i exp(-cR) sin(bR).  The reference evaluates exp(ikR)/(4piR) - 1/(4piR)
    (assembly.cu:73-77, bem_core.py:894-906); the two agree to the rounding
    noise of the reference's form, which is ~1e-16/(4 pi R) at coincident
    points."""
    k = complex(k)
    b, c = k.real, k.imag
    R = np.asarray(R, dtype=np.float64)
    Rs = np.maximum(R, 1e-300)
    sh = np.sin(0.5 * b * R)
    re = np.expm1(-c * R) * np.cos(b * R) - 2.0 * sh * sh
    im = np.exp(-c * R) * np.sin(b * R)
    zero = R == 0.0
    re = np.where(zero, -c, re / Rs)
    im = np.where(zero, b, im / Rs)
    return (re + 1j * im) * INV4PI


def _regular_LK(Ht, Hs, k, row_block=None, distance="direct", smooth="literal"):
    """Quadrature part of L and K for one (test half, source half) pair
    (assembly.cu:14-135 in FP64, bem_core.py:870-933).

    ``distance="direct"`` forms R = |r_t - r_s| (what the CUDA kernels do);
    ``distance="expanded"`` replays bem_core.py:888-891 literally,
    R^2 = |r_t|^2 + |r_s|^2 - 2 r_t.r_s by a matrix product.

    ``smooth="literal"`` takes G_smooth = exp(ik R_s)/(4 pi R_s) - 1/(4 pi R_s)
    with R_s = max(R, 1e-15) on same-triangle pairs, as the reference does
    (assembly.cu:63-77, bem_core.py:892-906); ``smooth="exact"`` uses the
    cancellation-free ``g_smooth``.  At coincident points (R = 0) the literal
    form returns Re = 0 when exp(ik R_s) rounds to 1 and +-1 ulp of
    1/(4 pi 1e-15) = +-0.0156 when it does not, instead of the limit
    -Im(k)/(4 pi); the expanded distance leaves R ~ 1e-8 at some coincident
    points, giving ~1e-16/(4 pi R) of noise there.  Lossless media: all forms
    agree to ~1e-10 relative.  Absorbing media: the literal forms differ from
    each other by the +-1 ulp term (~1e-4 relative on the diagonal blocks)."""
    Nt, Nq, _ = Ht.qp.shape
    Ns = Hs.qp.shape[0]
    L = np.zeros((Nt, Ns), dtype=complex)
    K = np.zeros((Nt, Ns), dtype=complex)
    ik = 1j * k
    ik_inv = 1j / k
    sq = Hs.qp.reshape(Ns * Nq, 3)
    sf = Hs.f.reshape(Ns * Nq, 3)
    sjw = Hs.jw.reshape(Ns * Nq)
    stri = np.repeat(Hs.tri, Nq)
    sqxsf = np.cross(sq, sf)
    bs = row_block or max(1, min(Nt, int(2.5e7 // max(1, Ns * Nq * Nq))))
    for b0 in range(0, Nt, bs):
        b1 = min(Nt, b0 + bs)
        B = b1 - b0
        tp = Ht.qp[b0:b1].reshape(B * Nq, 3)
        tf = Ht.f[b0:b1].reshape(B * Nq, 3)
        tjw = Ht.jw[b0:b1].reshape(B * Nq)
        ttri = np.repeat(Ht.tri[b0:b1], Nq)
        if distance == "expanded":
            R = (np.sum(tp ** 2, axis=1)[:, None] + np.sum(sq ** 2, axis=1)[None, :]
                 - 2.0 * (tp @ sq.T))
            R = np.sqrt(np.maximum(R, 0.0))
        else:
            d = tp[:, None, :] - sq[None, :, :]
            R = np.sqrt(np.sum(d * d, axis=-1))
        Rs = np.maximum(R, 1e-15)
        inv4piR = INV4PI / Rs
        G = np.exp(ik * Rs) * inv4piR
        sing = ttri[:, None] == stri[None, :]
        if smooth == "exact":
            Gu = np.where(sing, g_smooth(k, R), G)
        else:
            Gu = G - sing * inv4piR
        jw = tjw[:, None] * sjw[None, :]
        Gjw = Gu * jw
        fdot = tf @ sf.T
        Lv = (fdot * Gjw).reshape(B, Nq, Ns, Nq).sum(axis=(1, 3))
        Ls = Gjw.reshape(B, Nq, Ns, Nq).sum(axis=(1, 3))
        L[b0:b1] = ik * Lv - ik_inv * (Ht.div[b0:b1, None] * Hs.div[None, :]) * Ls
        valid = (~sing) & (R > 1e-12)
        gc = np.where(valid, (ik - 1.0 / Rs) / Rs, 0.0)
        triple = np.cross(tf, tp) @ sf.T - tf @ sqxsf.T
        K[b0:b1] = (G * gc * jw * triple).reshape(B, Nq, Ns, Nq).sum(axis=(1, 3))
    return L, K


def assemble_L_K(rwg, verts, tris, k, quad_order=7, distance="direct", smooth="literal"):
    """L and K (N x N, complex128, symmetric) for wavenumber k.

    L = sum over the four half pairs of the quadrature part, plus the
    same-triangle Graglia correction, then (L + L^T)/2; K likewise without a
    correction (assembly.cu:328-505, bem_core.py:787-1025)."""
    H = halves(rwg, verts, tris, quad_order)
    N = rwg["N"]
    L = np.zeros((N, N), dtype=complex)
    K = np.zeros((N, N), dtype=complex)
    if distance == "expanded":
        # bem_core.py:837-937 literally: passes (p,p), (p,m), (m,m) with its
        # batch size; the (m,p) pass is the transpose of (p,m).  The expanded
        # R^2 is not bitwise symmetric, so the pass structure matters there.
        Nq = H[0].qp.shape[1]
        bs = max(1, min(N, int(3e9 / max(1, N * Nq * Nq * 100))))
        for a, b in ((0, 0), (0, 1), (1, 1)):
            l, kk = _regular_LK(H[a], H[b], k, row_block=bs, distance=distance, smooth=smooth)
            if a != b:
                l = l + l.T
                kk = kk + kk.T
            L += l
            K += kk
    else:
        for a in range(2):
            for b in range(2):
                l, kk = _regular_LK(H[a], H[b], k, distance=distance, smooth=smooth)
                L += l
                K += kk
    L += singular_corrections(rwg, verts, tris, k, quad_order)
    return (L + L.T) / 2, (K + K.T) / 2


def pmchwt_blocks(L_ext, K_ext, L_int, K_int, eta_ext, eta_int):
    """Z = [[eta_e L_e + eta_i L_i, -(K_e+K_i)], [K_e+K_i, L_e/eta_e + L_i/eta_i]]
    (pmchwt.cu:36-51, bem_core.py:1060-1068)."""
    N = L_ext.shape[0]
    Ks = K_ext + K_int
    Z = np.zeros((2 * N, 2 * N), dtype=complex)
    Z[:N, :N] = eta_ext * L_ext + eta_int * L_int
    Z[:N, N:] = -Ks
    Z[N:, :N] = Ks
    Z[N:, N:] = L_ext / eta_ext + L_int / eta_int
    return Z


def assemble_pmchwt(rwg, verts, tris, k_ext, k_int, eta_ext, eta_int, quad_order=7,
                    distance="direct", smooth="literal"):
    """Row-major 2N x 2N PMCHWT matrix (pmchwt.cu:6-56, bem_core.py:1032-1068)."""
    Le, Ke = assemble_L_K(rwg, verts, tris, k_ext, quad_order, distance, smooth)
    Li, Ki = assemble_L_K(rwg, verts, tris, k_int, quad_order, distance, smooth)
    return pmchwt_blocks(Le, Ke, Li, Ki, eta_ext, eta_int)


def physics(ka, m):
    """k_ext = ka (unit radius), k_int = k_ext m, eta_ext = 1,
    eta_int = 1/|m| (main.cpp:192-196)."""
    m = complex(m)
    return complex(ka, 0.0), complex(ka, 0.0) * m, 1.0, 1.0 / abs(m)


# ---------------------------------------------------------------------------
# a9. Plane-wave right-hand side
# ---------------------------------------------------------------------------

def rhs_planewave(rwg, verts, tris, k_ext, eta_ext, E0, k_hat, quad_order=7):
    """b = [<f, E_inc>; <f, H_inc>], H0 = k_hat x E0 / eta_ext, phase
    exp(i k k_hat.r) (rhs.cpp:6-64, bem_core.py:1190-1219)."""
    E0 = np.asarray(E0, dtype=np.float64)
    k_hat = np.asarray(k_hat, dtype=np.float64)
    H0 = np.cross(k_hat, E0) / eta_ext
    N = rwg["N"]
    b = np.zeros(2 * N, dtype=complex)
    for h in halves(rwg, verts, tris, quad_order):
        ph = np.exp(1j * k_ext * np.einsum('i,nqi->nq', k_hat, h.qp))
        b[:N] += np.sum(np.einsum('nqi,i->nq', h.f, E0) * ph * h.jw, axis=1)
        b[N:] += np.sum(np.einsum('nqi,i->nq', h.f, H0) * ph * h.jw, axis=1)
    return b


# ---------------------------------------------------------------------------
# a10. Orientation quadrature
# ---------------------------------------------------------------------------

def euler_rotation(alpha, beta, gamma):
    """R = Rz(alpha) Ry(beta) Rz(gamma) (orient.cpp:4-36)."""
    ca, sa = math.cos(alpha), math.sin(alpha)
    cb, sb = math.cos(beta), math.sin(beta)
    cg, sg = math.cos(gamma), math.sin(gamma)
    Rz1 = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1.0]])
    Ry = np.array([[cb, 0, sb], [0, 1.0, 0], [-sb, 0, cb]])
    Rz2 = np.array([[cg, -sg, 0], [sg, cg, 0], [0, 0, 1.0]])
    return Rz1 @ (Ry @ Rz2)


def gauss_legendre(n):
    """Gauss-Legendre nodes/weights on [-1,1] by Newton from the Tricomi guess
    (orient.cpp:39-70)."""
    nodes, weights = np.zeros(n), np.zeros(n)
    for i in range(n):
        x = math.cos(math.pi * (i + 0.75) / (n + 0.5))
        for _ in range(100):
            p0, p1 = 1.0, x
            for j in range(2, n + 1):
                p0, p1 = p1, ((2 * j - 1) * x * p1 - (j - 1) * p0) / j
            dp = n * (x * p1 - p0) / (x * x - 1.0)
            dx = -p1 / dp
            x += dx
            if abs(dx) < 1e-15:
                break
        p0, p1 = 1.0, x
        for j in range(2, n + 1):
            p0, p1 = p1, ((2 * j - 1) * x * p1 - (j - 1) * p0) / j
        dp = n * (x * p1 - p0) / (x * x - 1.0)
        nodes[i] = x
        weights[i] = 2.0 / ((1.0 - x * x) * dp * dp)
    return nodes, weights


def generate_orientations(n_alpha, n_beta, n_gamma, beta_sym=1, gamma_sym=1,
                          gamma_mirror=False):
    """List of (RT, weight), ordered alpha-major then beta then gamma
    (orient.cpp:73-125)."""
    if beta_sym == 2:
        fn, fw = gauss_legendre(2 * n_beta)
        sel = fn > 0
        mu, mw = fn[sel], fw[sel] * 2.0
    else:
        mu, mw = gauss_legendre(n_beta)
    d_alpha = 2.0 * math.pi / n_alpha
    d_gamma = 2.0 * math.pi / n_gamma
    eff = gamma_sym * 2 if gamma_mirror else gamma_sym
    g_step = 2.0 * math.pi / (eff * n_gamma)
    out = []
    for ia in range(n_alpha):
        alpha = ia * d_alpha
        for ib in range(len(mu)):
            beta = math.acos(mu[ib])
            for ig in range(n_gamma):
                gamma = (ig + 0.5) * g_step if gamma_mirror else ig * g_step
                R = euler_rotation(alpha, beta, gamma)
                out.append((R.T.copy(), d_alpha * mw[ib] * d_gamma / (8.0 * math.pi ** 2)))
    return out


# ---------------------------------------------------------------------------
# a11. Dense LU and multi-RHS solve (LAPACK via SciPy, as the reference)
# ---------------------------------------------------------------------------

def lu_solve_dense(Z, B):
    """X = Z^-1 B by zgetrf/zgetrs (bem_core.py:1637, 1713; the GPU reference
    calls the same LAPACK routines in cuSOLVER, solver.cu:87-142)."""
    from scipy.linalg import lu_factor, lu_solve
    return lu_solve(lu_factor(Z), B)


# ---------------------------------------------------------------------------
# f4. GMRES on the dense Z with the reference's preconditioners
# ---------------------------------------------------------------------------

def aext_matrix(L_ext, K_ext, eta_ext):
    """A_ext = [[eta L_ext, -K_ext], [K_ext, L_ext / eta]]
    (build_aext_preconditioner, bem_core.py:1071-1090)."""
    N = L_ext.shape[0]
    A = np.zeros((2 * N, 2 * N), dtype=complex)
    A[:N, :N] = eta_ext * L_ext
    A[:N, N:] = -K_ext
    A[N:, :N] = K_ext
    A[N:, N:] = L_ext / eta_ext
    return A


def precond_solver(Z, kind, A_ext=None):
    """x -> M^-1 x for the preconditioners of solve_gmres (bem_core.py:1141-1166):
    'aext' (LU of A_ext), 'block_diag' (LU of Z11 and Z22), 'diag', None."""
    from scipy.linalg import lu_factor, lu_solve
    n = Z.shape[0]
    if kind == "aext":
        lu = lu_factor(A_ext)
        return lambda x: lu_solve(lu, x)
    if kind == "block_diag":
        N = n // 2
        lu11, lu22 = lu_factor(Z[:N, :N]), lu_factor(Z[N:, N:])

        def apply(x):
            y = np.empty(n, dtype=complex)
            y[:N] = lu_solve(lu11, x[:N])
            y[N:] = lu_solve(lu22, x[N:])
            return y
        return apply
    if kind == "diag":
        d = np.diag(Z).copy()
        return lambda x: x / d
    return lambda x: np.array(x, dtype=complex, copy=True)


def _zlartg(f, g):
    """LAPACK zlartg: c real, s complex, [c s; -conj(s) c] [f; g] = [r; 0],
    r with the phase of f."""
    if g == 0:
        return 1.0, 0j, f
    if f == 0:
        ag = abs(g)
        return 0.0, np.conj(g) / ag, complex(ag)
    af, ag = abs(f), abs(g)
    d = math.hypot(af, ag)
    ph = f / af
    return af / d, ph * np.conj(g) / d, ph * d


def gmres(A, b, psolve, rtol=1e-5, restart=20, maxiter=None):
    """scipy.sparse.linalg.gmres as the reference calls it (solve_gmres_aext,
    bem_core.py:1093-1123; solve_gmres :1126-1183), restated from SciPy 1.18.1
    scipy/sparse/linalg/_isolve/iterative.py (gmres): x0 = 0, left
    preconditioning (the preconditioned residual is minimised), modified
    Gram-Schmidt, Givens rotations by LAPACK lartg, inner loop ended by the
    adaptive ptol of gh-8400, restart cycles until ||b - A x|| <= rtol ||b||.
    Returns (x, info, inner_iterations)."""
    n = len(b)
    bnrm2 = np.linalg.norm(b)
    atol = rtol * bnrm2
    x = np.zeros(n, dtype=complex)
    if bnrm2 == 0:
        return np.array(b, dtype=complex), 0, 0
    eps = np.finfo(np.float64).eps
    maxiter = n * 10 if maxiter is None else maxiter
    restart = min(restart, n)
    Mb_nrm2 = np.linalg.norm(psolve(b))
    ptol_max_factor = 1.0
    ptol = Mb_nrm2 * min(ptol_max_factor, atol / bnrm2)
    presid = 0.0
    v = np.empty((restart + 1, n), dtype=complex)
    h = np.zeros((restart, restart + 1), dtype=complex)
    givens = np.zeros((restart, 2), dtype=complex)
    inner = 0
    rnorm = bnrm2
    r = np.array(b, dtype=complex)
    if np.linalg.norm(r) < atol:
        return x, 0, 0
    for _ in range(maxiter):
        v[0] = psolve(r)
        tmp = np.linalg.norm(v[0])
        v[0] *= 1 / tmp
        S = np.zeros(restart + 1, dtype=complex)
        S[0] = tmp
        breakdown = False
        for col in range(restart):
            w = psolve(A @ v[col])
            h0 = np.linalg.norm(w)
            for k in range(col + 1):
                t = np.vdot(v[k], w)
                h[col, k] = t
                w -= t * v[k]
            h1 = np.linalg.norm(w)
            h[col, col + 1] = h1
            v[col + 1] = w
            if h1 <= eps * h0:
                h[col, col + 1] = 0
                breakdown = True
            else:
                v[col + 1] *= 1 / h1
            for k in range(col):
                c, s = givens[k, 0], givens[k, 1]
                n0, n1 = h[col, k], h[col, k + 1]
                h[col, k], h[col, k + 1] = c * n0 + s * n1, -np.conj(s) * n0 + c * n1
            c, s, mag = _zlartg(h[col, col], h[col, col + 1])
            givens[col] = c, s
            h[col, col], h[col, col + 1] = mag, 0
            t = -np.conj(s) * S[col]
            S[col], S[col + 1] = c * S[col], t
            presid = abs(t)
            inner += 1
            if presid <= ptol or breakdown:
                break
        if h[col, col] == 0:
            S[col] = 0
        y = np.array(S[:col + 1])
        for k in range(col, 0, -1):
            if y[k] != 0:
                y[k] /= h[k, k]
                y[:k] -= y[k] * h[k, :k]
        if y[0] != 0:
            y[0] /= h[0, 0]
        x += y @ v[:col + 1]
        r = b - A @ x
        rnorm = np.linalg.norm(r)
        if rnorm <= atol or breakdown:
            break
        if presid <= ptol:
            ptol_max_factor = max(eps, 0.25 * ptol_max_factor)
        else:
            ptol_max_factor = min(1.0, 1.5 * ptol_max_factor)
        ptol = presid * min(ptol_max_factor, atol / rnorm)
    return x, (0 if rnorm <= atol else maxiter), inner


# ---------------------------------------------------------------------------
# a12-a14. Far field and Mueller matrix
# ---------------------------------------------------------------------------

class FarFieldCache:
    """Quadrature points, basis values and weights of both halves
    (farfield.cu:9-52): arrays of shape (2, N, Nq, ...)."""

    def __init__(self, rwg, verts, tris, quad_order=7):
        H = halves(rwg, verts, tris, quad_order)
        self.qp = np.stack([h.qp for h in H])
        self.f = np.stack([h.f for h in H])
        self.jw = np.stack([h.jw for h in H])
        self.N = rwg["N"]


def far_field_vec(cache, cJ, cM, k_ext, eta_ext, r_hats, sM=-1.0):
    """F(r_hat) = -ik/(4pi) (eta J_perp + sM r_hat x M) for coefficient
    vectors cJ, cM (N,) and directions r_hats (D, 3) -> (D, 3) complex
    (farfield.cu:100-262 / :351-431, bem_core.py:1265-1294)."""
    r_hats = np.asarray(r_hats, dtype=np.float64)
    ph = np.exp(-1j * k_ext * np.einsum('di,hnqi->dhnq', r_hats, cache.qp))
    w = ph * cache.jw[None]                                    # (D,2,N,Nq)
    integ = np.einsum('dhnq,hnqi->dhni', w, cache.f)           # (D,2,N,3)
    Jt = np.einsum('dhni,n->di', integ, cJ)
    Mt = np.einsum('dhni,n->di', integ, cM)
    Jp = Jt - r_hats * np.sum(r_hats * Jt, axis=1, keepdims=True)
    Mc = np.cross(r_hats, Mt)
    return -1j * k_ext / (4 * math.pi) * (eta_ext * Jp + sM * Mc)


def amplitude_to_mueller(S1, S2, S3, S4):
    """Bohren & Huffman eq. 3.16 (farfield.cu:464-508, bem_core.py:1407-1438);
    returns (4, 4, ntheta)."""
    a1, a2, a3, a4 = (np.abs(S) ** 2 for S in (S1, S2, S3, S4))
    s23 = S2 * np.conj(S3)
    s14 = S1 * np.conj(S4)
    s24 = S2 * np.conj(S4)
    s13 = S1 * np.conj(S3)
    s12 = S1 * np.conj(S2)
    s34 = S3 * np.conj(S4)
    s21 = S2 * np.conj(S1)
    s42 = S4 * np.conj(S2)
    s43 = S4 * np.conj(S3)
    M = np.zeros((4, 4, len(S1)))
    M[0, 0] = 0.5 * (a1 + a2 + a3 + a4)
    M[0, 1] = 0.5 * (a2 - a1 + a4 - a3)
    M[0, 2] = s23.real + s14.real
    M[0, 3] = s23.imag - s14.imag
    M[1, 0] = 0.5 * (a2 - a1 - a4 + a3)
    M[1, 1] = 0.5 * (a2 + a1 - a4 - a3)
    M[1, 2] = s23.real - s14.real
    M[1, 3] = s23.imag + s14.imag
    M[2, 0] = s24.real + s13.real
    M[2, 1] = s24.real - s13.real
    M[2, 2] = s12.real + s34.real
    M[2, 3] = s21.imag + s43.imag
    M[3, 0] = s42.imag + s13.imag
    M[3, 1] = s42.imag - s13.imag
    M[3, 2] = s12.imag - s34.imag
    M[3, 3] = s12.real - s34.real
    return M


def theta_grid(ntheta):
    """theta_i = pi i/(ntheta-1) (main.cpp:331-333)."""
    return np.pi * np.arange(ntheta) / (ntheta - 1)


def lab_frame(theta):
    """r_hat = (sin t, 0, cos t), e_theta = (cos t, 0, -sin t), e_phi = y
    (main.cpp:766-771)."""
    st, ct = np.sin(theta), np.cos(theta)
    z = np.zeros_like(theta)
    return (np.stack([st, z, ct], 1), np.stack([ct, z, -st], 1),
            np.array([0.0, 1.0, 0.0]))


def mueller_from_solutions(cache, X, orients, k_ext, eta_ext, theta,
                           gamma_mirror=False):
    """Weighted orientation sum of Mueller matrices from solution columns
    X[:, 2o] (par) and X[:, 2o+1] (perp) (main.cpp:757-846)."""
    N = cache.N
    r_lab, et_lab, ep_lab = lab_frame(theta)
    Mavg = np.zeros((4, 4, len(theta)))
    ik = -1j * k_ext
    k2 = abs(k_ext) ** 2
    for o, (RT, w) in enumerate(orients):
        rh = r_lab @ RT.T
        ep = et_lab @ RT.T
        epp = RT @ ep_lab
        Fpar = far_field_vec(cache, X[:N, 2 * o], X[N:, 2 * o], k_ext, eta_ext, rh)
        Fperp = far_field_vec(cache, X[:N, 2 * o + 1], X[N:, 2 * o + 1], k_ext, eta_ext, rh)
        S2 = ik * np.sum(Fpar * ep, axis=1)
        S4 = ik * (Fpar @ epp)
        S3 = ik * np.sum(Fperp * ep, axis=1)
        S1 = ik * (Fperp @ epp)
        M = amplitude_to_mueller(S1, S2, S3, S4)
        if gamma_mirror:
            M.reshape(16, -1)[[2, 3, 6, 7, 8, 9, 12, 13]] = 0.0
        Mavg += w * M / k2
    return Mavg


def orientation_rhs(rwg, verts, tris, orients, k_ext, eta_ext, quad_order=7):
    """Columns [par_0, perp_0, par_1, ...]: k_hat = RT z, e_par = RT x,
    e_perp = RT y (main.cpp:739-751, bem_core.py:1660-1700)."""
    N = rwg["N"]
    B = np.zeros((2 * N, 2 * len(orients)), dtype=complex)
    for o, (RT, _) in enumerate(orients):
        kh = RT @ np.array([0.0, 0.0, 1.0])
        B[:, 2 * o] = rhs_planewave(rwg, verts, tris, k_ext, eta_ext, RT[:, 0], kh, quad_order)
        B[:, 2 * o + 1] = rhs_planewave(rwg, verts, tris, k_ext, eta_ext, RT[:, 1], kh, quad_order)
    return B


def single_orientation_mueller(rwg, verts, tris, Z, k_ext, eta_ext, ntheta=181,
                               quad_order=7):
    """--single: k_hat = z, E = x (par) and y (perp); phi = 0 plane
    (main.cpp:671-718, bem_core.py:1330-1456)."""
    orients = [(np.eye(3), 1.0)]
    B = orientation_rhs(rwg, verts, tris, orients, k_ext, eta_ext, quad_order)
    X = lu_solve_dense(Z, B)
    cache = FarFieldCache(rwg, verts, tris, quad_order)
    return mueller_from_solutions(cache, X, orients, k_ext, eta_ext,
                                  theta_grid(ntheta)), X, B


def orientation_average_mueller(rwg, verts, tris, Z, k_ext, eta_ext, n_alpha,
                                n_beta, n_gamma, ntheta=181, quad_order=7):
    """Batched orientation average (main.cpp:720-846,
    bem_core.py:1606-1767)."""
    orients = generate_orientations(n_alpha, n_beta, n_gamma)
    B = orientation_rhs(rwg, verts, tris, orients, k_ext, eta_ext, quad_order)
    X = lu_solve_dense(Z, B)
    cache = FarFieldCache(rwg, verts, tris, quad_order)
    return mueller_from_solutions(cache, X, orients, k_ext, eta_ext,
                                  theta_grid(ntheta)), X, B
