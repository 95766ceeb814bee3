// Host harness around the library's rest-state set-up
// (cpu-ipc_b200/csrc/scene_setup.cpp: surface extraction, material, rest
// shapes, masses, bending data, bbox-relative scalars) for
// tests/test_scene_setup.py.
#include "scene_setup.h"

#include <cstring>
#include <exception>

static cipc::SceneRest R;

extern "C" int ss_setup(int nv, const double* x, int nt, const int* tets, int nf, const int* tris, const double* tetE,
                        const double* p, int bending, const double* bbMin, const double* bbMax) {
    cipc::SceneInput in;
    in.nv = nv; in.nt = nt; in.nf = nf;
    in.x.assign(x, x + 3 * (size_t)nv);
    in.tets.assign(tets, tets + 4 * (size_t)nt);
    in.tris.assign(tris, tris + 3 * (size_t)nf);
    if (tetE) in.tetE.assign(tetE, tetE + nt);
    in.density = p[0]; in.cloth_density = p[1]; in.thickness = p[2]; in.E = p[3]; in.nu = p[4];
    in.clothE = p[5]; in.shearE = p[6]; in.bendE = p[7]; in.strainRate = p[8]; in.relDhat = p[9];
    in.quadBending = bending == 1;
    in.hingeBending = bending == 2;
    for (int k = 0; k < 3; ++k) { in.bboxMin[k] = bbMin[k]; in.bboxMax[k] = bbMax[k]; }
    try {
        R = cipc::SceneRest();
        cipc::setupScene(in, R);
    } catch (const std::exception&) {
        return 1;
    }
    return 0;
}

static const std::vector<double>* dvec(int which) {
    switch (which) {
    case 0: return &R.mass; case 1: return &R.DmInv; case 2: return &R.vol; case 3: return &R.DmInv2;
    case 4: return &R.area; case 5: return &R.bendQ; case 6: return &R.hingeW; case 7: return &R.hingeTh0;
    case 8: return &R.tetMu; case 9: return &R.tetLam; default: return nullptr;
    }
}
static const std::vector<int>* ivec(int which) {
    switch (which) {
    case 20: return &R.bendV; case 21: return &R.faces; case 22: return &R.surfVerts; case 23: return &R.edges;
    default: return nullptr;
    }
}

extern "C" long long ss_size(int which) {
    if (auto d = dvec(which)) return (long long)d->size();
    if (auto i = ivec(which)) return (long long)i->size();
    return -1;
}

extern "C" void ss_get(int which, void* out) {
    if (auto d = dvec(which)) std::memcpy(out, d->data(), d->size() * sizeof(double));
    else if (auto i = ivec(which)) std::memcpy(out, i->data(), i->size() * sizeof(int));
}

// lengthRate, volumeRate, stretchS, shearS, plateRigidity, meanMass, avgEdge, bboxDiag2, Hhat, Fhat, dTol
extern "C" void ss_scalars(double* o) {
    const double v[11] = {R.lengthRate, R.volumeRate, R.stretchS, R.shearS, R.plateRigidity, R.meanMass,
                          R.avgEdge, R.bboxDiag2, R.Hhat, R.Fhat, R.dTol};
    std::memcpy(o, v, sizeof(v));
}
