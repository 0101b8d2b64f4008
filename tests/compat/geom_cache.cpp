// The device-geometry cache behind the reference's per-call surface:
// compute_rhs_planewave on six distinct meshes (more than the four unused
// geometries the library keeps), on the first mesh again, and on that mesh
// with one vertex moved (same sizes and connectivity, other content); the
// far-field cache uploaded for two meshes in turn.  Writes each result for
// the test to compare with the library's own RHS / far field of each mesh.
//
// Usage: geom_cache OUTDIR
#include <complex>
#include <cstdio>
#include <string>
#include <vector>

#include "farfield.h"
#include "mesh.h"
#include "rhs.h"
#include "rwg.h"

using cd = std::complex<double>;

static bool dump(const std::string& path, const std::vector<cd>& v) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = std::fwrite(v.data(), sizeof(cd), v.size(), f) == v.size();
    return std::fclose(f) == 0 && ok;
}

static std::vector<cd> rhs(const Mesh& m) {
    RWG r = build_rwg(m);
    std::vector<cd> b(2 * (size_t)r.N);
    compute_rhs_planewave(r, m, cd(2.0, 0.0), 1.0, Vec3(1, 0, 0), Vec3(0, 0, 1), 7, b.data());
    return b;
}

static std::vector<cd> farfield(const Mesh& m) {
    RWG r = build_rwg(m);
    FFCache c;
    c.init(r, m, 7);
    FFCacheGPU g;
    g.upload(c);
    std::vector<cd> J(2 * (size_t)r.N), M(2 * (size_t)r.N);
    for (int n = 0; n < r.N; n++) J[n] = cd(1.0 / (1 + n), 0.5), M[n] = cd(0.25, -1.0 / (2 + n));
    const int ndir = 5;
    std::vector<double> rh(3 * ndir);
    for (int d = 0; d < ndir; d++) rh[3 * d] = 0.6 * d / ndir, rh[3 * d + 1] = 0.0, rh[3 * d + 2] = 1.0;
    std::vector<cd> Fv(2 * (size_t)ndir * 3);
    compute_farfield_batch_cuda(g, J.data(), M.data(), rh.data(), cd(2.0, 0.0), 1.0, 2, 1, ndir, Fv.data());
    return Fv;
}

int main(int argc, char** argv) {
    if (argc < 2) return 1;
    const std::string out = argv[1];
    std::vector<Mesh> meshes = {icosphere(1.0, 1), hex_prism(1.3, 1), icosphere(0.7, 1),
                                hex_prism(0.8, 1),  icosphere(1.0, 2), hex_prism(1.5, 2)};
    for (size_t i = 0; i < meshes.size(); i++)
        if (!dump(out + "/rhs" + std::to_string(i) + ".bin", rhs(meshes[i]))) return 2;
    if (!dump(out + "/rhs0_again.bin", rhs(meshes[0]))) return 3;
    Mesh moved = meshes[0];
    moved.verts[0] = moved.verts[0] * 1.05;
    if (!dump(out + "/rhs0_moved.bin", rhs(moved))) return 4;
    if (!dump(out + "/ff0.bin", farfield(meshes[0])) || !dump(out + "/ff1.bin", farfield(meshes[1])) ||
        !dump(out + "/ff0_again.bin", farfield(meshes[0])))
        return 5;
    std::printf("geom_cache: done\n");
    return 0;
}
