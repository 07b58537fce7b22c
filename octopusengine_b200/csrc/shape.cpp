// Shape-function derivatives and quadrature rules of the supported elements.
//
// Tetrahedra are written over barycentric coordinates L = (1-x-y-z, x, y, z) with
// dL/dX = (-1,-1,-1), e_x, e_y, e_z, and differentiated in closed form by the chain rule:
//   P1 corner    N = L_i                      dN = dL_i
//   P2 corner    N = L_i (2 L_i - 1)          dN = (4 L_i - 1) dL_i
//   P2 edge ij   N = 4 L_i L_j                dN = 4 (L_j dL_i + L_i dL_j)
//   P3 corner    N = (3L-1)(3L-2)L / 2        dN = (27 L^2 - 18 L + 2)/2 dL_i
//   P3 edge i->j N = 9/2 L_i L_j (3 L_i - 1)  (node one third of the way from i to j)
//   P3 face ijk  N = 27 L_i L_j L_k
// Hexahedra are tensor products of 1-D Lagrange bases on [-1, 1].  The node numbering,
// quadrature points and weights are those of the reference's FEM_Shape classes
// (octopus/include/Dynamic/FEM/FEM_Shape.h: Tetra_4 :36-66, Hexa_8 :175-224,
// Tetra_10 :227-272, Tetra_20 :274-482 with the 11-point polyfem rule, Hexa_27 :483-690).
#include <cmath>

#include "host.hpp"

namespace octb {

int element_nodes(int e) {
    switch (e) {
        case kTetra: return 4; case kHexa: return 8; case kTetra10: return 10;
        case kTetra20: return 20; case kHexa27: return 27; default: return -1;
    }
}
int element_quadrature(int e) {
    switch (e) {
        case kTetra: return 1; case kHexa: return 8; case kTetra10: return 4;
        case kTetra20: return 11; case kHexa27: return 27; default: return -1;
    }
}

namespace {

// The 11-point tetrahedron rule used by the reference for Tetra_20 (published with
// polyfem); weights are for the unit reference tetrahedron before the 1/6 volume factor.
const double kT20Points[11][3] = {
    {0.040490506727590428, 0.013560701879802881, 0.77125473269537614},
    {0.75250850700965499, 0.068099370938206658, 0.097987203649279112},
    {0.067223294893383398, 0.035183929773598716, 0.15636389323939529},
    {0.41926631387951302, 0.047781435559086663, 0.47961101102565507},
    {0.45076587609127683, 0.059456616299433829, 0.056824017127933668},
    {0.12941137378891041, 0.33019041483746447, 0.0023910074574393647},
    {0.12154199133392780, 0.30649398842969028, 0.56297276014304609},
    {0.097204644587583267, 0.68439041545304002, 0.11180076739738309},
    {0.029569495206479612, 0.31790356021339461, 0.32329398483747895},
    {0.43271023904776856, 0.35382323920929709, 0.10962240533194123},
    {0.24027666492807262, 0.12680172591539202, 0.32847320672203845}};
const double kT20Weights[11] = {
    0.039251090924839957, 0.055273369155936898, 0.055393798871576368, 0.059933185146559528,
    0.069469965937635367, 0.076162715245558357, 0.079426680068025307, 0.10646803415549010,
    0.11023423242849766, 0.15497611601624608, 0.19341081204963445};

// Node tables in the reference numbering.
const int kP2Edges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
const int kP3Edges[12][2] = {{0, 1}, {1, 0}, {1, 2}, {2, 1}, {2, 0}, {0, 2},
                             {0, 3}, {3, 0}, {1, 3}, {3, 1}, {2, 3}, {3, 2}};
const int kP3Faces[4][3] = {{0, 1, 3}, {1, 2, 3}, {0, 2, 3}, {0, 1, 2}};
const int kHexNodes[27][3] = {
    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1},
    {0, -1, -1}, {1, 0, -1}, {0, 1, -1}, {-1, 0, -1}, {-1, -1, 0}, {1, -1, 0}, {1, 1, 0}, {-1, 1, 0},
    {0, -1, 1}, {1, 0, 1}, {0, 1, 1}, {-1, 0, 1}, {0, 0, -1}, {0, -1, 0}, {1, 0, 0}, {0, 1, 0},
    {-1, 0, 0}, {0, 0, 1}, {0, 0, 0}};

const double kDL[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

// 1-D quadratic Lagrange basis on nodes {-1, 0, 1} and its derivative.
double lag(int node, double s) {
    if (node < 0) return 0.5 * s * (s - 1.0);
    if (node > 0) return 0.5 * s * (s + 1.0);
    return (1.0 - s) * (1.0 + s);
}
double dlag(int node, double s) {
    if (node < 0) return s - 0.5;
    if (node > 0) return s + 0.5;
    return -2.0 * s;
}

void tet_derivatives(int e, const double* x, double* dN) {
    const double L[4] = {1.0 - x[0] - x[1] - x[2], x[0], x[1], x[2]};
    auto put = [&](int node, int a, double ca, int b = -1, double cb = 0, int c = -1, double cc = 0) {
        for (int k = 0; k < 3; ++k) {
            double v = ca * kDL[a][k];
            if (b >= 0) v += cb * kDL[b][k];
            if (c >= 0) v += cc * kDL[c][k];
            dN[node * 3 + k] = v;
        }
    };
    if (e == kTetra) {
        for (int i = 0; i < 4; ++i) put(i, i, 1.0);
    } else if (e == kTetra10) {
        for (int i = 0; i < 4; ++i) put(i, i, 4.0 * L[i] - 1.0);
        for (int k = 0; k < 6; ++k) {
            const int i = kP2Edges[k][0], j = kP2Edges[k][1];
            put(4 + k, i, 4.0 * L[j], j, 4.0 * L[i]);
        }
    } else {
        for (int i = 0; i < 4; ++i) put(i, i, 0.5 * (27.0 * L[i] * L[i] - 18.0 * L[i] + 2.0));
        for (int k = 0; k < 12; ++k) {
            const int i = kP3Edges[k][0], j = kP3Edges[k][1];
            // N = 4.5 L_i L_j (3 L_i - 1)
            put(4 + k, i, 4.5 * L[j] * (6.0 * L[i] - 1.0), j, 4.5 * L[i] * (3.0 * L[i] - 1.0));
        }
        for (int k = 0; k < 4; ++k) {
            const int i = kP3Faces[k][0], j = kP3Faces[k][1], l = kP3Faces[k][2];
            put(16 + k, i, 27.0 * L[j] * L[l], j, 27.0 * L[i] * L[l], l, 27.0 * L[i] * L[j]);
        }
    }
}

void hex_derivatives(int e, const double* x, double* dN) {
    const int ne = e == kHexa ? 8 : 27;
    for (int i = 0; i < ne; ++i) {
        const int* n = kHexNodes[i];
        if (e == kHexa) {
            const double a = 1.0 + n[0] * x[0], b = 1.0 + n[1] * x[1], c = 1.0 + n[2] * x[2];
            dN[i * 3 + 0] = 0.125 * n[0] * b * c;
            dN[i * 3 + 1] = 0.125 * a * n[1] * c;
            dN[i * 3 + 2] = 0.125 * a * b * n[2];
        } else {
            const double lx = lag(n[0], x[0]), ly = lag(n[1], x[1]), lz = lag(n[2], x[2]);
            dN[i * 3 + 0] = dlag(n[0], x[0]) * ly * lz;
            dN[i * 3 + 1] = lx * dlag(n[1], x[1]) * lz;
            dN[i * 3 + 2] = lx * ly * dlag(n[2], x[2]);
        }
    }
}

}  // namespace

// Shape-function values at reference coordinates x (FEM_Shape::build_shape), same bases as
// the derivatives above.
bool shape_values(int e, const double* x, double* N) {
    if (e == kTetra || e == kTetra10 || e == kTetra20) {
        const double L[4] = {1.0 - x[0] - x[1] - x[2], x[0], x[1], x[2]};
        if (e == kTetra) {
            for (int i = 0; i < 4; ++i) N[i] = L[i];
        } else if (e == kTetra10) {
            for (int i = 0; i < 4; ++i) N[i] = L[i] * (2.0 * L[i] - 1.0);
            for (int k = 0; k < 6; ++k) N[4 + k] = 4.0 * L[kP2Edges[k][0]] * L[kP2Edges[k][1]];
        } else {
            for (int i = 0; i < 4; ++i) N[i] = 0.5 * (3.0 * L[i] - 1.0) * (3.0 * L[i] - 2.0) * L[i];
            for (int k = 0; k < 12; ++k) {
                const double li = L[kP3Edges[k][0]], lj = L[kP3Edges[k][1]];
                N[4 + k] = 4.5 * li * lj * (3.0 * li - 1.0);
            }
            for (int k = 0; k < 4; ++k) N[16 + k] = 27.0 * L[kP3Faces[k][0]] * L[kP3Faces[k][1]] * L[kP3Faces[k][2]];
        }
        return true;
    }
    if (e == kHexa || e == kHexa27) {
        const int ne = e == kHexa ? 8 : 27;
        for (int i = 0; i < ne; ++i) {
            const int* n = kHexNodes[i];
            N[i] = e == kHexa ? 0.125 * (1.0 + n[0] * x[0]) * (1.0 + n[1] * x[1]) * (1.0 + n[2] * x[2])
                              : lag(n[0], x[0]) * lag(n[1], x[1]) * lag(n[2], x[2]);
        }
        return true;
    }
    return false;
}

// Reference-element node coordinates (FEM_Shape::get_vertices for the corners; edge and face
// nodes where the node tables put them).
bool reference_nodes(int e, double* X) {
    const double tc[4][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    auto put = [&](int node, double a, int i, double b, int j, double c = 0, int k = 0) {
        for (int d = 0; d < 3; ++d) X[3 * node + d] = a * tc[i][d] + b * tc[j][d] + c * tc[k][d];
    };
    if (e == kTetra || e == kTetra10 || e == kTetra20) {
        for (int i = 0; i < 4; ++i) put(i, 1.0, i, 0.0, i);
        if (e == kTetra10)
            for (int k = 0; k < 6; ++k) put(4 + k, 0.5, kP2Edges[k][0], 0.5, kP2Edges[k][1]);
        if (e == kTetra20) {
            for (int k = 0; k < 12; ++k) put(4 + k, 2.0 / 3.0, kP3Edges[k][0], 1.0 / 3.0, kP3Edges[k][1]);
            for (int k = 0; k < 4; ++k) put(16 + k, 1.0 / 3.0, kP3Faces[k][0], 1.0 / 3.0, kP3Faces[k][1], 1.0 / 3.0, kP3Faces[k][2]);
        }
        return true;
    }
    if (e == kHexa || e == kHexa27) {
        const int ne = e == kHexa ? 8 : 27;
        for (int i = 0; i < ne; ++i)
            for (int d = 0; d < 3; ++d) X[3 * i + d] = kHexNodes[i][d];
        return true;
    }
    return false;
}

bool shape_table(int e, ShapeTable& s) {
    s = ShapeTable();
    s.ne = element_nodes(e);
    s.nq = element_quadrature(e);
    if (s.ne < 0) return false;
    switch (e) {
        case kTetra: s.qp = {0.25, 0.25, 0.25}; s.w = {1.0 / 6.0}; break;
        case kHexa: {
            const double c = 1.0 / std::sqrt(3.0);
            for (int q = 0; q < 8; ++q) for (int k = 0; k < 3; ++k) s.qp.push_back(c * kHexNodes[q][k]);
            s.w.assign(8, 1.0);
            break;
        }
        case kTetra10: {
            const double a = (5.0 - std::sqrt(5.0)) / 20.0, b = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0;
            s.qp = {b, a, a, a, b, a, a, a, b, a, a, a};
            s.w.assign(4, 1.0 / 24.0);
            break;
        }
        case kTetra20:
            for (int q = 0; q < 11; ++q) {
                for (int k = 0; k < 3; ++k) s.qp.push_back(kT20Points[q][k]);
                s.w.push_back(kT20Weights[q] / 6.0);
            }
            break;
        case kHexa27: {
            // Gauss-Legendre 3x3x3 at +-sqrt(3/5) and 0, listed in the node order above
            const double v = std::sqrt(0.6);
            for (int q = 0; q < 27; ++q) {
                double w = 1.0;
                for (int k = 0; k < 3; ++k) {
                    s.qp.push_back(v * kHexNodes[q][k]);
                    w *= kHexNodes[q][k] == 0 ? 8.0 / 9.0 : 5.0 / 9.0;
                }
                s.w.push_back(w);
            }
            break;
        }
    }
    s.dN.assign((size_t)s.nq * s.ne * 3, 0.0);
    for (int q = 0; q < s.nq; ++q) {
        double* d = &s.dN[(size_t)q * s.ne * 3];
        if (e == kHexa || e == kHexa27) hex_derivatives(e, &s.qp[3 * q], d);
        else tet_derivatives(e, &s.qp[3 * q], d);
    }
    return true;
}

}  // namespace octb
