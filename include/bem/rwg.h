// Reference-compatible RWG basis (BEM-CPP src/rwg.h:7-18).
#ifndef BEM_COMPAT_RWG_H
#define BEM_COMPAT_RWG_H

#include <vector>

#include "mesh.h"

struct RWG {
    int N;
    std::vector<int> tri_p, tri_m;
    std::vector<Vec3> free_p, free_m;
    std::vector<double> length, area_p, area_m;
};

RWG build_rwg(const Mesh& mesh);

#endif
