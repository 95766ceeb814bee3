// Host-side rest-state set-up of a GPU context (see scene_setup.cpp).
#pragma once

#include <vector>

namespace cipc {

struct SceneInput {
    int nv = 0, nt = 0, nf = 0;
    std::vector<double> x;
    std::vector<int> tets, tris;
    std::vector<double> tetE;
    double density = 1000, cloth_density = 200, thickness = 1e-3, E = 1e4, nu = 0.49, clothE = 1e4, shearE = 10, bendE = 1e4, strainRate = 100;
    double relDhat = 1e-3;
    bool quadBending = true;
    bool hingeBending = false;  // dihedral-angle hinges instead (the reference's build without USE_QUADRATIC_BENDING)
    double bboxMin[3] = {0, 0, 0}, bboxMax[3] = {0, 0, 0};
    bool hasSurface = false;
    std::vector<int> faces, surfVerts, edges;
};

struct SceneRest {
    double lengthRate = 0, volumeRate = 0, stretchS = 0, shearS = 0, plateRigidity = 0;
    double meanMass = 0, avgEdge = 0, bboxDiag2 = 0, Hhat = 0, Fhat = 0, dTol = 0;
    std::vector<double> mass, DmInv, vol, tetMu, tetLam, DmInv2, area, bendQ;
    std::vector<double> hingeW, hingeTh0;  // per hinge: rest weight l0^2 / (2 A0 + 2 A1), rest angle
    std::vector<int> bendV, faces, surfVerts, edges;
};

void materialFromYoung(double E, double nu, double& lengthRate, double& volumeRate);
void setupScene(const SceneInput& in, SceneRest& out);

}  // namespace cipc
