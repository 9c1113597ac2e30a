// quadrature.cpp -- velocity sphere of the reference: the subdivided icosahedron
// with flat-triangle Voronoi weights (icosahedron.h:36-171, Point.h:64-69,
// wrapped by gen_v2d_icosahedron, CartGrid.cpp:46-61).
//
// N = 10*nn^2 + 2 unit vectors.  Each of the 10 rhombic patches spanned by
// four icosahedron vertices is refined bilinearly into nn x nn cells and
// projected to the sphere; every cell is split into two triangles and each
// vertex collects, per triangle, the areas of the two sub-triangles spanned
// with the circumcentre.  The weights sum to ~4*pi*(0.93..0.995), not 1; the
// solver uses them as the reference does.  The floating-point operations are
// performed in the reference's order, so the result is bit-identical to it.
#include <cmath>
#include <vector>

namespace nuosc {
namespace {

struct V3 {
    double x, y, z;
};
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 scale(double k, V3 a) { return {k * a.x, k * a.y, k * a.z}; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double norm2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
double norm(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

V3 circumcenter(V3 A, V3 B, V3 C) {
    const V3 n = cross(sub(B, A), sub(C, A));
    const V3 AC = sub(C, A), AB = sub(B, A);
    return add(A, scale(0.5 / norm2(n), cross(n, sub(scale(norm2(AC), AB), scale(norm2(AB), AC)))));
}

// vertices (a, b, c, d) of the 10 patches; the same table as icosahedron.h:39-40
constexpr unsigned kPatch[10][4] = {{1, 0, 2, 6}, {6, 2, 7, 11}, {2, 0, 3, 7}, {7, 3, 8, 11}, {3, 0, 4, 8},
                                    {8, 4, 9, 11}, {4, 0, 5, 9}, {9, 5, 10, 11}, {5, 0, 1, 10}, {10, 1, 6, 11}};

}  // namespace

int icosahedron_count(int nn) { return 10 * nn * nn + 2; }

void icosahedron(int nn_, std::vector<double> &vx, std::vector<double> &vy, std::vector<double> &vz,
                 std::vector<double> &vw) {
    const unsigned nn = unsigned(nn_), NP = 5, N = 2 * NP * nn * nn + 2, W = nn + 1;
    const double lambda = 1.10714871779409;  // latitude of the upper ring (atan 2)
    V3 base[12];
    for (unsigned i = 1; i <= NP; ++i) {
        base[i] = {std::cos(2 * i * M_PI / NP) * std::sin(lambda), std::sin(2 * i * M_PI / NP) * std::sin(lambda),
                   std::cos(lambda)};
        base[i + NP] = {std::cos((2 * i + 1) * M_PI / NP) * std::sin(lambda),
                        std::sin((2 * i + 1) * M_PI / NP) * std::sin(lambda), -base[i].z};
    }
    base[0] = {0, 0, 1};
    base[11] = {0, 0, -1};

    std::vector<V3> X(N);
    X[0] = base[0];
    X[N - 1] = base[11];
    for (unsigned p = 0; p < 2 * NP; ++p) {
        const V3 A = base[kPatch[p][0]], B = base[kPatch[p][1]], C = base[kPatch[p][2]], D = base[kPatch[p][3]];
        for (unsigned i = 0; i < nn; ++i)
            for (unsigned j = 0; j < nn; ++j) {
                const V3 q = add(scale(double(i), add(scale(double(j), C), scale(double(nn - j), D))),
                                 scale(double(nn - i), add(scale(double(j), B), scale(double(nn - j), A))));
                X[p * nn * nn + i * nn + j + 1] = scale(1.0 / norm(q), q);
            }
    }

    // lattice (p, i, j), i,j in [0, nn], -> unique point id; the patch edges
    // i == nn or j == nn belong to the neighbouring patches or a pole
    std::vector<unsigned> id(2 * NP * W * W, 0);
    auto at = [&](unsigned p, unsigned i, unsigned j) -> unsigned & { return id[(p * W + i) * W + j]; };
    for (unsigned p = 0; p < 2 * NP; ++p) {
        for (unsigned i = 0; i < nn; ++i)
            for (unsigned j = 0; j < nn; ++j) at(p, i, j) = p * nn * nn + i * nn + j + 1;
        if (p == 2 * NP - 1) {
            for (unsigned i = 1; i <= nn; ++i) {
                at(p, i - 1, nn) = 1 + nn * (i - 1);
                at(p, nn, i) = 2 * nn * nn - (nn - 1) - nn * (i - 1);
            }
            at(p, nn, 0) = N - 1;
        } else if (p % 2 == 1) {
            for (unsigned i = 1; i <= nn; ++i) {
                at(p, i - 1, nn) = (p + 1) * nn * nn + 1 + nn * (i - 1);
                at(p, nn, i) = (p + 3) * nn * nn - (nn - 1) - nn * (i - 1);
            }
            at(p, nn, 0) = N - 1;
        } else {
            for (unsigned i = 1; i <= nn; ++i) {
                at(p, i, nn) = ((p + 2) * nn * nn + (nn - i) + 1) % (2 * NP * nn * nn);
                at(p, nn, i - 1) = (p + 1) * nn * nn + i;
            }
            at(p, 0, nn) = 0;
        }
    }

    vw.assign(N, 0.0);
    for (unsigned p = 0; p < 2 * NP; ++p)
        for (unsigned i = 0; i < nn; ++i)
            for (unsigned j = 0; j < nn; ++j) {
                const unsigned iA = at(p, i, j), iC = at(p, i + 1, j + 1);
                const unsigned iBs[2] = {at(p, i, j + 1), at(p, i + 1, j)};
                for (unsigned iB : iBs) {
                    const V3 A = X[iA], Bp = X[iB], C = X[iC];
                    const V3 O = circumcenter(A, Bp, C);
                    const double fAB = norm(scale(0.25, cross(sub(O, A), sub(Bp, A))));
                    const double fBC = norm(scale(0.25, cross(sub(O, Bp), sub(C, Bp))));
                    const double fCA = norm(scale(0.25, cross(sub(O, C), sub(A, C))));
                    vw[iA] += fAB + fCA;
                    vw[iB] += fBC + fAB;
                    vw[iC] += fCA + fBC;
                }
            }
    vx.resize(N);
    vy.resize(N);
    vz.resize(N);
    for (unsigned k = 0; k < N; ++k) {
        vx[k] = X[k].x;
        vy[k] = X[k].y;
        vz[k] = X[k].z;
    }
}

}  // namespace nuosc
