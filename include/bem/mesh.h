// Reference-compatible mesh interface (BEM-CPP src/mesh.h:7-44).
#ifndef BEM_COMPAT_MESH_H
#define BEM_COMPAT_MESH_H

#include <vector>

#include "types.h"

struct Mesh {
    std::vector<Vec3> verts;
    std::vector<int> tris;  // 3 vertex indices per triangle
    int nv() const { return (int)verts.size(); }
    int nt() const { return (int)tris.size() / 3; }
    void tri_verts(int ti, Vec3& v0, Vec3& v1, Vec3& v2) const {
        v0 = verts[tris[3 * ti]];
        v1 = verts[tris[3 * ti + 1]];
        v2 = verts[tris[3 * ti + 2]];
    }
    double tri_area(int ti) const {
        Vec3 v0, v1, v2;
        tri_verts(ti, v0, v1, v2);
        return 0.5 * (v1 - v0).cross(v2 - v0).norm();
    }
};

Mesh icosphere(double radius, int refinements);
Mesh hex_prism(double aspect_ratio, int refinements);
Mesh load_obj(const char* filename);
Mesh subdivide_flat(const Mesh& m);
double mesh_volume(const Mesh& m);
double normalize_mesh(Mesh& m);
double mesh_dmax(const Mesh& m);

#endif
