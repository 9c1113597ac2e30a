/*
 * nuosc_oracle.c -- CPU restatement of nuosc's RK4 time step (TEST INFRASTRUCTURE ONLY).
 *
 * This file is the oracle: a plain-C, double-precision restatement of the
 * reference's hot path, used only by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the checker.  Nothing in the product
 * (nuosc_b200/) links or calls it.
 *
 * Parity is pinned: tests/test_oracle_vs_ref.py checks this restatement
 * against the reference's own CPU code compiled by oracle/Makefile
 * (oracle/_ref/), and tests/golden/ holds fixtures generated from that build.
 *
 * Reference files restated (paths inside chunyulin/nuosc):
 *   icosahedron.h:36-171, Point.h:64-69   velocity quadrature (Voronoi weights)
 *   CartGrid.cpp:191-208, CartGrid.h:91    geometry and ghosted index
 *   nuosc_init.cpp:8-10,70-130             initial data (seeded epsilon injected)
 *   nuosc_init.cpp:11-14,24-68             "NOC" initial data (ipt 4; seeded phases, every x)
 *   nuosc_init.cpp:162-230                 advection tests (ipt 10 Advtest, 20 Square, 30 Triangle)
 *   nuosc_ana.cpp:58-61,121                the advection test's integrals I1, I2
 *   nuosc_boundary.cpp:4-52                periodic ghost fill
 *   nuosc_class.cpp:11-307                 calRHS (moments, commutator, ADV, KO, vacuum)
 *   nuosc_class.cpp:313-372,374-427        vectorize and step_rk4
 *   nuosc_ana.cpp:3-137                    eval_conserved / analysis
 *
 * Field order everywhere: 0 ee, 1 mm, 2 emr, 3 emi, 4 bee, 5 bmm, 6 bemr, 7 bemi
 * (FieldVar::getAllFields, nuosc_class.h:58-65).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#define NF 8

/* ------------------------------------------------------------------ */
/* Velocity quadrature: subdivided icosahedron with flat-triangle      */
/* Voronoi weights (icosahedron.h:36-171, Point.h:64-69).              */
/* ------------------------------------------------------------------ */
typedef struct { double x, y, z; } pt;

static pt p_add(pt a, pt b) { pt r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static pt p_sub(pt a, pt b) { pt r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static pt p_scale(double k, pt a) { pt r = {k * a.x, k * a.y, k * a.z}; return r; }
static pt p_cross(pt a, pt b) {
    pt r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static double p_norm2(pt a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static double p_norm(pt a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

/* circumcenter of triangle ABC in 3D (Point.h:64-69) */
static pt circumcenter(pt A, pt B, pt C) {
    pt ABxAC = p_cross(p_sub(B, A), p_sub(C, A));
    pt AC = p_sub(C, A);
    pt AB = p_sub(B, A);
    pt t = p_sub(p_scale(p_norm2(AC), AB), p_scale(p_norm2(AB), AC));
    return p_add(A, p_scale(0.5 / p_norm2(ABxAC), p_cross(ABxAC, t)));
}

int orc_nv(int nn) { return 10 * nn * nn + 2; }

/* Corner indices (A,B,C,D) of the 10 rhombic patches of the icosahedron
 * (the IB table of icosahedron.h:39-40; the table itself must be identical). */
static const unsigned PATCH[40] = {1, 0, 2, 6,  6, 2, 7, 11, 2, 0, 3, 7,  7, 3, 8, 11,
                                   3, 0, 4, 8,  8, 4, 9, 11, 4, 0, 5, 9,  9, 5, 10, 11,
                                   5, 0, 1, 10, 10, 1, 6, 11};

void orc_icosahedron(int nn_, double *vx, double *vy, double *vz, double *vw) {
    const unsigned NP = 5, nn = (unsigned)nn_;
    const double lambda = 1.10714871779409; /* icosahedron.h:41 */
    const unsigned N = 2 * NP * nn * nn + 2;
    pt bp[12];
    for (unsigned i = 1; i <= NP; ++i) { /* icosahedron.h:51-58 */
        bp[i].x = cos(2 * i * M_PI / NP) * sin(lambda);
        bp[i].y = sin(2 * i * M_PI / NP) * sin(lambda);
        bp[i].z = cos(lambda);
        bp[i + NP].x = cos((2 * i + 1) * M_PI / NP) * sin(lambda);
        bp[i + NP].y = sin((2 * i + 1) * M_PI / NP) * sin(lambda);
        bp[i + NP].z = -bp[i].z;
    }
    bp[0].x = 0; bp[0].y = 0; bp[0].z = 1;
    bp[2 * NP + 1].x = 0; bp[2 * NP + 1].y = 0; bp[2 * NP + 1].z = -1;

    pt *X = (pt *)calloc(N, sizeof(pt));
    X[0] = bp[0];
    X[N - 1] = bp[2 * NP + 1];
    for (unsigned p = 0; p < 2 * NP; ++p) { /* icosahedron.h:67-81 */
        unsigned a = PATCH[4 * p], b = PATCH[4 * p + 1], c = PATCH[4 * p + 2], d = PATCH[4 * p + 3];
        for (int i = 0; i < (int)nn; ++i)
            for (int j = 0; j < (int)nn; ++j) {
                unsigned pij = p * nn * nn + i * nn + j + 1;
                pt q = p_add(p_scale((double)i, p_add(p_scale((double)j, bp[c]), p_scale((double)(nn - j), bp[d]))),
                             p_scale((double)(nn - i), p_add(p_scale((double)j, bp[b]), p_scale((double)(nn - j), bp[a]))));
                double iL = 1.0 / p_norm(q);
                X[pij] = p_scale(iL, q);
            }
    }

    /* unique-point index of each patch's (nn+1)^2 lattice (icosahedron.h:107-135) */
    const unsigned W = nn + 1;
    unsigned *ui = (unsigned *)calloc(2 * NP * W * W, sizeof(unsigned));
#define FID(p, i, j) (((p) * W + (i)) * W + (j))
    for (unsigned p = 0; p < 2 * NP; ++p) {
        for (unsigned i = 0; i < nn; ++i)
            for (unsigned j = 0; j < nn; ++j) ui[FID(p, i, j)] = p * nn * nn + i * nn + j + 1;
        if (p == 2 * NP - 1) {
            for (unsigned i = 1; i <= nn; ++i) {
                ui[FID(p, i - 1, nn)] = 1 + nn * (i - 1);
                ui[FID(p, nn, i)] = 2 * nn * nn - (nn - 1) - nn * (i - 1);
            }
            ui[FID(p, nn, 0)] = N - 1;
        } else if (p % 2 == 1) {
            for (unsigned i = 1; i <= nn; ++i) {
                ui[FID(p, i - 1, nn)] = (p + 1) * nn * nn + 1 + nn * (i - 1);
                ui[FID(p, nn, i)] = (p + 3) * nn * nn - (nn - 1) - nn * (i - 1);
            }
            ui[FID(p, nn, 0)] = N - 1;
        } else {
            for (unsigned i = 1; i <= nn; ++i) {
                ui[FID(p, i, nn)] = ((p + 2) * nn * nn + (nn - i) + 1) % (2 * NP * nn * nn);
                ui[FID(p, nn, i - 1)] = (p + 1) * nn * nn + i;
            }
            ui[FID(p, 0, nn)] = 0;
        }
    }

    /* Voronoi area accumulation (icosahedron.h:137-170) */
    for (unsigned k = 0; k < N; ++k) vw[k] = 0.0;
    for (unsigned p = 0; p < 2 * NP; ++p)
        for (unsigned i = 0; i < nn; ++i)
            for (unsigned j = 0; j < nn; ++j) {
                unsigned iA = ui[FID(p, i, j)], iC = ui[FID(p, i + 1, j + 1)];
                pt A = X[iA], C = X[iC];
                for (int tri = 0; tri < 2; ++tri) {
                    unsigned iB = tri == 0 ? ui[FID(p, i, j + 1)] : ui[FID(p, i + 1, j)];
                    pt B = X[iB];
                    pt O = circumcenter(A, B, C);
                    double fAB = p_norm(p_scale(0.25, p_cross(p_sub(O, A), p_sub(B, A))));
                    double fBC = p_norm(p_scale(0.25, p_cross(p_sub(O, B), p_sub(C, B))));
                    double fCA = p_norm(p_scale(0.25, p_cross(p_sub(O, C), p_sub(A, C))));
                    vw[iA] += fAB + fCA;
                    vw[iB] += fBC + fAB;
                    vw[iC] += fCA + fBC;
                }
            }
#undef FID
    for (unsigned k = 0; k < N; ++k) { vx[k] = X[k].x; vy[k] = X[k].y; vz[k] = X[k].z; }
    free(ui);
    free(X);
}

/* ------------------------------------------------------------------ */
/* Seeded perturbation: one uniform draw in [0,1) per (x,z) cell,      */
/* replacing the reference's rand() (nuosc_init.cpp:5,100).            */
/* ------------------------------------------------------------------ */
static uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double orc_uniform(uint64_t seed, int i, int j) {
    uint64_t key = ((uint64_t)(uint32_t)i << 32) | (uint64_t)(uint32_t)j;
    return (double)(mix64(mix64(seed) ^ key) >> 11) * 0x1.0p-53;
}

/* ------------------------------------------------------------------ */
/* Simulation object: ghosted layout (CartGrid.h:91) and 4 registers   */
/* (v_stat, v_rhs, v_pre, v_cor) as in NuOsc (nuosc_class.h:108).      */
/* ------------------------------------------------------------------ */
typedef struct orc_sim {
    int nx, nz, nv, gx, gz;
    double x0, x1, z0, z1, dx, dz, dt, ds_L, ko, mu, pmo, phy_time;
    double *vx, *vy, *vz, *vw;
    double *G0, *G0b; /* per velocity (the generic init makes them x,z independent) */
    double n_nue0[2];
    long lpts;
    double *reg[4][NF]; /* 0 stat, 1 rhs, 2 pre, 3 cor */
    double *noc_phi;    /* explicit ipt = 4 phases (orc_set_noc_phases), or NULL: seeded */
    int noc_nphi;
    int xoff;           /* x-slab: global index of plane 0 (seeded ipt = 1 draws) */
} orc_sim;

static inline long gidx(const orc_sim *s, int i, int j, int v) {
    return ((long)(i + s->gx) * (s->nz + 2 * s->gz) + j + s->gz) * s->nv + v;
}

/* nx = int((x1-x0)/dx) as in CartGrid.cpp:196-197 */
void orc_geometry(double x0, double x1, double z0, double z1, double dx, double dz, int *nx, int *nz) {
    *nx = (int)((x1 - x0) / dx);
    *nz = (int)((z1 - z0) / dz);
}

orc_sim *orc_create(int nn, double x0, double x1, double z0, double z1, double dx, double dz,
                    double cfl, double ko, int ghost, double mu, double pmo) {
    orc_sim *s = (orc_sim *)calloc(1, sizeof(orc_sim));
    s->x0 = x0; s->x1 = x1; s->z0 = z0; s->z1 = z1; s->dx = dx; s->dz = dz;
    orc_geometry(x0, x1, z0, z1, dx, dz, &s->nx, &s->nz);
    s->gx = s->gz = ghost;
    s->nv = orc_nv(nn);
    s->ko = ko; s->mu = mu; s->pmo = pmo;
    s->dt = dz * cfl;                                /* nuosc_class.cpp:464 */
    s->ds_L = dx * dz / (z1 - z0) / (x1 - x0);       /* nuosc_class.cpp:461 */
    s->phy_time = 0.0;
    s->vx = (double *)malloc(sizeof(double) * s->nv);
    s->vy = (double *)malloc(sizeof(double) * s->nv);
    s->vz = (double *)malloc(sizeof(double) * s->nv);
    s->vw = (double *)malloc(sizeof(double) * s->nv);
    s->G0 = (double *)calloc(s->nv, sizeof(double));
    s->G0b = (double *)calloc(s->nv, sizeof(double));
    orc_icosahedron(nn, s->vx, s->vy, s->vz, s->vw);
    s->lpts = (long)(s->nx + 2 * s->gx) * (s->nz + 2 * s->gz) * s->nv;
    for (int r = 0; r < 4; ++r)
        for (int f = 0; f < NF; ++f) s->reg[r][f] = (double *)calloc(s->lpts, sizeof(double));
    return s;
}

void orc_destroy(orc_sim *s) {
    if (!s) return;
    for (int r = 0; r < 4; ++r)
        for (int f = 0; f < NF; ++f) free(s->reg[r][f]);
    free(s->vx); free(s->vy); free(s->vz); free(s->vw); free(s->G0); free(s->G0b);
    free(s->noc_phi);
    free(s);
}

void orc_info(const orc_sim *s, int *ints, double *dbls) {
    ints[0] = s->nx; ints[1] = s->nz; ints[2] = s->nv; ints[3] = s->gx;
    dbls[0] = s->dt; dbls[1] = s->ds_L; dbls[2] = s->phy_time; dbls[3] = s->n_nue0[0]; dbls[4] = s->n_nue0[1];
}
void orc_velocities(const orc_sim *s, double *vx, double *vy, double *vz, double *vw, double *G0, double *G0b) {
    memcpy(vx, s->vx, sizeof(double) * s->nv); memcpy(vy, s->vy, sizeof(double) * s->nv);
    memcpy(vz, s->vz, sizeof(double) * s->nv); memcpy(vw, s->vw, sizeof(double) * s->nv);
    memcpy(G0, s->G0, sizeof(double) * s->nv); memcpy(G0b, s->G0b, sizeof(double) * s->nv);
}

/* angular spectrum g(vx,vz) (nuosc_init.cpp:8-10) */
static double gspec(double vx, double vz, double sx, double sz) {
    return exp(-(vx - 1.0) * (vx - 1.0) / (2.0 * sx * sx) - (vz - 1.0) * (vz - 1.0) / (2.0 * sz * sz));
}

/*
 * Initial data, generic branch of fillInitValue (nuosc_init.cpp:70-130).
 * ipt 0: Gaussian in z (eps_c), 1: seeded uniform eps0*U(-1,1) per (x,z),
 * 2: eps_p profile, 3: constant eps0.  lnuex/lnuebx <= 0 mean "infinite"
 * (the reference default DBL_MAX, nuosc.cpp:36-37).
 */
static void fill_noc(orc_sim *s, double alpha, double lnue, double lnueb, uint64_t seed);
static void fill_advtest(orc_sim *s, int ipt, double eps0, double sigma);

void orc_fill_init(orc_sim *s, int ipt, double alpha, double eps0, double sigma, double lnue,
                   double lnueb, double lnuex, double lnuebx, uint64_t seed) {
    if (ipt == 4) { fill_noc(s, alpha, lnue, lnueb, seed); return; }
    if (ipt >= 10) { fill_advtest(s, ipt, eps0, sigma); return; }
    if (lnuex <= 0) lnuex = DBL_MAX;
    if (lnuebx <= 0) lnuebx = DBL_MAX;
    double ing0 = 0, ing1 = 0;
    double *ng = (double *)malloc(sizeof(double) * s->nv), *ngb = (double *)malloc(sizeof(double) * s->nv);
    for (int v = 0; v < s->nv; ++v) {
        ng[v] = gspec(s->vx[v], s->vz[v], lnuex, lnue);
        ngb[v] = gspec(s->vx[v], s->vz[v], lnuebx, lnueb);
        ing0 += s->vw[v] * ng[v];
        ing1 += s->vw[v] * ngb[v];
    }
    ing0 = 1.0 / ing0;
    ing1 = 1.0 / ing1;
    for (int v = 0; v < s->nv; ++v) {
        s->G0[v] = ng[v] * ing0;
        s->G0b[v] = alpha * ngb[v] * ing1;
    }
    double n00 = 0, n01 = 0;
    double **st = s->reg[0];
    for (int i = 0; i < s->nx; ++i)
        for (int j = 0; j < s->nz; ++j) {
            double Zj = s->z0 + (j + 0.5) * s->dz; /* CartGrid.cpp:200 */
            double tmpr;
            if (ipt == 0) tmpr = eps0 * exp(-(Zj) * (Zj) / (2.0 * sigma * sigma));
            else if (ipt == 1) tmpr = eps0 * (2.0 * orc_uniform(seed, s->xoff + i, j) - 1.0);
            else if (ipt == 2) tmpr = eps0 * (1.0 + cos(2 * M_PI * (Zj) / (2.0 * sigma * sigma))) * 0.5;
            else tmpr = eps0;
            double p3o = sqrt(1.0 - tmpr * tmpr);
            for (int v = 0; v < s->nv; ++v) {
                long k = gidx(s, i, j, v);
                double G = s->G0[v], Gb = s->G0b[v];
                st[0][k] = 0.5 * G * (1.0 + p3o);
                st[1][k] = 0.5 * G * (1.0 - p3o);
                st[2][k] = 0.5 * G * tmpr;
                st[3][k] = 0.0;
                st[4][k] = 0.5 * Gb * (1.0 + p3o);
                st[5][k] = 0.5 * Gb * (1.0 - p3o);
                st[6][k] = 0.5 * Gb * tmpr;
                st[7][k] = 0.0;
                n00 += s->vw[v] * st[0][k];
                n01 += s->vw[v] * st[4][k];
            }
        }
    s->n_nue0[0] = n00 * s->ds_L;
    s->n_nue0[1] = n01 * s->ds_L;
    s->phy_time = 0.0;
    free(ng); free(ngb);
}

/* Phases of the ipt = 4 initial data: n = 2 (nz/20) + 1 values (NULL: back
 * to the seeded phases).  Lets a test feed the reference's rand() phases. */
void orc_set_noc_phases(orc_sim *s, int n, const double *phi) {
    free(s->noc_phi);
    s->noc_phi = NULL;
    s->noc_nphi = 0;
    if (phi && n > 0) {
        s->noc_phi = (double *)malloc(sizeof(double) * n);
        memcpy(s->noc_phi, phi, sizeof(double) * n);
        s->noc_nphi = n;
    }
}

/* spectrum of the NOC branch: normalised over vz in [-1, 1] by erf (nuosc_init.cpp:11-14) */
static double gnoc(double v, double sigma) {
    const double v0 = 1.0;
    const double N = sigma * sqrt(0.5 * M_PI) * (erf((1.0 + v0) / sigma / sqrt(2.0)) + erf((1.0 - v0) / sigma / sqrt(2.0)));
    return exp(-(v - v0) * (v - v0) / (2.0 * sigma * sigma)) / N;
}

/*
 * ipt = 4, the "NOC" branch (nuosc_init.cpp:24-68), restated for every x (the
 * reference fills only the x = 0 column): amax = nz/20 modes k = -amax ..
 * amax-1, k != 0, of amplitude 1e-7/|k| and phase phi[k + amax], with
 * phi[m] = 2 pi U(seed, m, -1) unless explicit phases were set; P1, P2 =
 * their cos and sin sums, P3 = sqrt(1 - P1^2 - P2^2); bemi = -emi.  n_nue0
 * is set from the filled state (the reference leaves it unset here).
 */
static void fill_noc(orc_sim *s, double alpha, double lnue, double lnueb, uint64_t seed) {
    const int amax = s->nz / 2 / 10;
    double *phi = (double *)malloc(sizeof(double) * (2 * amax + 1));
    for (int m = 0; m <= 2 * amax; ++m)
        phi[m] = (s->noc_phi && m < s->noc_nphi) ? s->noc_phi[m] : 2.0 * M_PI * orc_uniform(seed, m, -1);
    for (int v = 0; v < s->nv; ++v) {
        s->G0[v] = gnoc(s->vz[v], lnue);
        s->G0b[v] = alpha * gnoc(s->vz[v], lnueb);
    }
    const double pi2oL = 2.0 * M_PI / (s->z0 - s->z1);
    double n00 = 0, n01 = 0;
    double **st = s->reg[0];
    for (int j = 0; j < s->nz; ++j) {
        const double Zj = s->z0 + (j + 0.5) * s->dz;
        double tr = 0.0, ti = 0.0;
        for (int k = -amax; k < amax; ++k) {
            if (k == 0) continue;
            tr += 1.e-7 / abs(k) * cos(pi2oL * k * Zj + phi[k + amax]);
            ti += 1.e-7 / abs(k) * sin(pi2oL * k * Zj + phi[k + amax]);
        }
        const double t2 = sqrt(1.0 - tr * tr - ti * ti);
        for (int i = 0; i < s->nx; ++i)
            for (int v = 0; v < s->nv; ++v) {
                const long q = gidx(s, i, j, v);
                const double G = s->G0[v], Gb = s->G0b[v];
                st[0][q] = 0.5 * G * (1.0 + t2);
                st[1][q] = 0.5 * G * (1.0 - t2);
                st[2][q] = 0.5 * G * tr;
                st[3][q] = 0.5 * G * ti;
                st[4][q] = 0.5 * Gb * (1.0 + t2);
                st[5][q] = 0.5 * Gb * (1.0 - t2);
                st[6][q] = 0.5 * Gb * tr;
                st[7][q] = -0.5 * Gb * ti;
                n00 += s->vw[v] * st[0][q];
                n01 += s->vw[v] * st[4][q];
            }
    }
    s->n_nue0[0] = n00 * s->ds_L;
    s->n_nue0[1] = n01 * s->ds_L;
    s->phy_time = 0.0;
    free(phi);
}

/*
 * ipt = 10 fillInitAdvtest, 20 fillInitSquare, 30 fillInitTriangle
 * (nuosc_init.cpp:162-230): G0 = G0b = 1, ee = the profile in z, the other
 * fields 0.  n_nue0 is set from the filled state.
 */
static void fill_advtest(orc_sim *s, int ipt, double eps0, double sigma) {
    for (int v = 0; v < s->nv; ++v) s->G0[v] = s->G0b[v] = 1.0;
    double n00 = 0;
    for (int j = 0; j < s->nz; ++j) {
        const double Z = s->z0 + (j + 0.5) * s->dz;
        double t = 0.0;
        if (ipt == 10) {
            const double sd = 0.33;
            t = exp(-(Z * Z) / (1.0 * sigma * sigma)) + ((Z + sd) * (Z + sd) <= sigma * sigma) +
                (int)(Z - sd < 0 && Z - sd > -sigma) * (sigma + Z - sd) / sigma +
                (int)(Z - sd >= 0 && Z - sd < sigma) * (sigma - Z + sd) / sigma;
            t = t * eps0;
        } else if (ipt == 20) {
            if (Z * Z <= sigma * sigma) t = eps0;
        } else {
            if (Z < 0 && Z > -sigma) t = (sigma + Z) * eps0 / sigma;
            else if (Z >= 0 && Z < sigma) t = (sigma - Z) * eps0 / sigma;
        }
        for (int i = 0; i < s->nx; ++i)
            for (int v = 0; v < s->nv; ++v) {
                const long q = gidx(s, i, j, v);
                s->reg[0][0][q] = t;
                for (int f = 1; f < NF; ++f) s->reg[0][f][q] = 0.0;
                n00 += s->vw[v] * t;
            }
    }
    s->n_nue0[0] = n00 * s->ds_L;
    s->n_nue0[1] = 0.0;
    s->phy_time = 0.0;
}

/* The advection test's integrals (nuosc_ana.cpp:58-61,121): I1 = sum w ee / nor,
 * I2 = sum w ee^2 / nor, nor = sum w G0 over all cells. */
void orc_adv_integrals(const orc_sim *s, double *out) {
    double I1 = 0, I2 = 0, nor = 0;
    for (int i = 0; i < s->nx; ++i)
        for (int j = 0; j < s->nz; ++j)
            for (int v = 0; v < s->nv; ++v) {
                const double ee = s->reg[0][0][gidx(s, i, j, v)];
                I1 += s->vw[v] * ee;
                I2 += s->vw[v] * ee * ee;
                nor += s->vw[v] * s->G0[v];
            }
    out[0] = I1 / nor;
    out[1] = I2 / nor;
}

/* Set G0/G0b directly (used with externally supplied state). */
void orc_set_g0(orc_sim *s, const double *G0, const double *G0b, double n0, double n1) {
    memcpy(s->G0, G0, sizeof(double) * s->nv);
    memcpy(s->G0b, G0b, sizeof(double) * s->nv);
    s->n_nue0[0] = n0; s->n_nue0[1] = n1;
}

void orc_set_state(orc_sim *s, int reg, int f, const double *compact) {
    for (int i = 0; i < s->nx; ++i)
        for (int j = 0; j < s->nz; ++j)
            memcpy(&s->reg[reg][f][gidx(s, i, j, 0)], &compact[((long)i * s->nz + j) * s->nv], sizeof(double) * s->nv);
}
void orc_get_state(const orc_sim *s, int reg, int f, double *compact) {
    for (int i = 0; i < s->nx; ++i)
        for (int j = 0; j < s->nz; ++j)
            memcpy(&compact[((long)i * s->nz + j) * s->nv], &s->reg[reg][f][gidx(s, i, j, 0)], sizeof(double) * s->nv);
}
void orc_set_time(orc_sim *s, double t) { s->phy_time = t; }

/* Periodic ghost fill, z first then x; corners untouched (nuosc_boundary.cpp:4-52). */
static void boundary_z(orc_sim *s, double **F) {
#pragma omp parallel for collapse(2)
    for (int i = 0; i < s->nx; ++i)
        for (int j = 0; j < s->gz; ++j)
            for (int v = 0; v < s->nv; ++v) {
                long l0 = gidx(s, i, -j - 1, v), l1 = gidx(s, i, s->nz - j - 1, v);
                long r0 = gidx(s, i, s->nz + j, v), r1 = gidx(s, i, j, v);
                for (int f = 0; f < NF; ++f) { F[f][l0] = F[f][l1]; F[f][r0] = F[f][r1]; }
            }
}

static void periodic_boundary(orc_sim *s, double **F) {
    boundary_z(s, F);
#pragma omp parallel for collapse(2)
    for (int i = 0; i < s->gx; ++i)
        for (int j = 0; j < s->nz; ++j)
            for (int v = 0; v < s->nv; ++v) {
                long l0 = gidx(s, -i - 1, j, v), l1 = gidx(s, s->nx - i - 1, j, v);
                long r0 = gidx(s, s->nx + i, j, v), r1 = gidx(s, i, j, v);
                for (int f = 0; f < NF; ++f) { F[f][l0] = F[f][l1]; F[f][r0] = F[f][r1]; }
            }
}

void orc_update_boundary(orc_sim *s, int reg) { periodic_boundary(s, s->reg[reg]); }

/*
 * out = L(in) on interior cells (nuosc_class.cpp:11-307), two-flavour path.
 * gx == 3 selects the 6th-difference KO (KO_ORD_3 undefined, :112-117),
 * gx == 2 the 4th-difference KO (KO_ORD_3 defined, :119-123).
 * Default 4th-order central advection (:179-183).  Vacuum term (:280-287)
 * with theta = 37 degrees (nuosc_class.h:120-122) scaled by pmo.
 */
static void calrhs(const orc_sim *s, double **out, double **in) {
    const int nv = s->nv;
    const long nzv = (long)nv * (s->nz + 2 * s->gz);
    const double mu = s->mu, pmo = s->pmo, ko = s->ko;
    const double theta = 37 * M_PI / 180.;
    const double ct = cos(2 * theta), st = sin(2 * theta);
    const int ko3 = (s->gx == 3);
    const double ko_eps_x = ko3 ? -ko / s->dx / 64.0 : -ko / s->dx / 16.0;
    const double ko_eps_z = ko3 ? -ko / s->dz / 64.0 : -ko / s->dz / 16.0;
    const double *vx = s->vx, *vy = s->vy, *vz = s->vz, *vw = s->vw;
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < s->nx; ++i)
        for (int j = 0; j < s->nz; ++j) {
            double emRm[4] = {0, 0, 0, 0}, emIp[4] = {0, 0, 0, 0}, eemm[4] = {0, 0, 0, 0};
            for (int k = 0; k < nv; ++k) { /* velocity moments, :62-82 */
                long ijk = gidx(s, i, j, k);
                const double v4[4] = {1, vx[k], vy[k], vz[k]};
                for (int q = 0; q < 4; ++q) {
                    emRm[q] += v4[q] * vw[k] * (in[6][ijk] - in[2][ijk]);
                    emIp[q] += v4[q] * vw[k] * (in[7][ijk] + in[3][ijk]);
                    eemm[q] += v4[q] * vw[k] * (in[4][ijk] - in[5][ijk] - in[0][ijk] + in[1][ijk]);
                }
            }
            for (int v = 0; v < nv; ++v) {
                long ijv = gidx(s, i, j, v);
                const double factor_x = -vx[v] / (12 * s->dx);
                const double factor_z = -vz[v] / (12 * s->dz);
                double rhs[NF];
                for (int f = 0; f < NF; ++f) {
                    const double *x = &in[f][ijv];
                    double adv = factor_z * ((x[-2 * nv] - x[2 * nv]) - 8.0 * (x[-nv] - x[nv])) +
                                 factor_x * ((x[-2 * nzv] - x[2 * nzv]) - 8.0 * (x[-nzv] - x[nzv]));
                    double kod;
                    if (ko3)
                        kod = ko_eps_z * (x[-3 * nv] + x[3 * nv] - 6 * (x[-2 * nv] + x[2 * nv]) + 15 * (x[-nv] + x[nv]) - 20 * x[0]) +
                              ko_eps_x * (x[-3 * nzv] + x[3 * nzv] - 6 * (x[-2 * nzv] + x[2 * nzv]) + 15 * (x[-nzv] + x[nzv]) - 20 * x[0]);
                    else
                        kod = ko_eps_z * (x[-2 * nv] + x[2 * nv] - 4 * (x[-nv] + x[nv]) + 6 * x[0]) +
                              ko_eps_x * (x[-2 * nzv] + x[2 * nzv] - 4 * (x[-nzv] + x[nzv]) + 6 * x[0]);
                    rhs[f] = adv + kod;
                }
                /* commutator with the self-interaction Hamiltonian, :187-200 */
                double iemRm = emRm[0] - emRm[1] * vx[v] - emRm[2] * vy[v] - emRm[3] * vz[v];
                double iemIp = emIp[0] - emIp[1] * vx[v] - emIp[2] * vy[v] - emIp[3] * vz[v];
                double ieemm = eemm[0] - eemm[1] * vx[v] - eemm[2] * vy[v] - eemm[3] * vz[v];
                const double ee = in[0][ijv], mm = in[1][ijv], emr = in[2][ijv], emi = in[3][ijv];
                const double bee = in[4][ijv], bmm = in[5][ijv], bemr = in[6][ijv], bemi = in[7][ijv];
                double Iee = 2 * mu * (emi * iemRm + emr * iemIp);
                double Iemr = -mu * ((ee - mm) * iemIp + ieemm * emi);
                double Iemi = mu * ((mm - ee) * iemRm + ieemm * emr);
                double Ibee = 2 * mu * (bemi * iemRm + bemr * iemIp);
                double Ibemr = -mu * ((bee - bmm) * iemIp + ieemm * bemi);
                double Ibemi = mu * ((bmm - bee) * iemRm + ieemm * bemr);
                /* vacuum term, :280-287 */
                out[0][ijv] = Iee + rhs[0] - pmo * 2 * st * emi;
                out[1][ijv] = -Iee + rhs[1] + pmo * 2 * st * emi;
                out[2][ijv] = Iemr + rhs[2] - pmo * 2 * ct * emi;
                out[3][ijv] = Iemi + rhs[3] + pmo * (2 * ct * emr + st * (ee - mm));
                out[4][ijv] = Ibee + rhs[4] - pmo * 2 * st * bemi;
                out[5][ijv] = -Ibee + rhs[5] + pmo * 2 * st * bemi;
                out[6][ijv] = Ibemr + rhs[6] - pmo * 2 * ct * bemi;
                out[7][ijv] = Ibemi + rhs[7] + pmo * (2 * ct * bemr + st * (bee - bmm));
            }
        }
}

/* v0 = v1 + a*v2 over the interior (nuosc_class.cpp:313-330) */
static void vec1(const orc_sim *s, double **v0, double **v1, double a, double **v2) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < s->nx; ++i)
        for (int j = 0; j < s->nz; ++j)
            for (int v = 0; v < s->nv; ++v) {
                long k = gidx(s, i, j, v);
                for (int f = 0; f < NF; ++f) v0[f][k] = v1[f][k] + a * v2[f][k];
            }
}
/* v0 = v1 + a*(v2 + v3) over the interior (nuosc_class.cpp:333-351) */
static void vec2(const orc_sim *s, double **v0, double **v1, double a, double **v2, double **v3) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < s->nx; ++i)
        for (int j = 0; j < s->nz; ++j)
            for (int v = 0; v < s->nv; ++v) {
                long k = gidx(s, i, j, v);
                for (int f = 0; f < NF; ++f) v0[f][k] = v1[f][k] + a * (v2[f][k] + v3[f][k]);
            }
}

/* calRHS(v_rhs, v_stat) after a periodic ghost fill of v_stat */
void orc_calrhs(orc_sim *s, int out_reg, int in_reg) {
    periodic_boundary(s, s->reg[in_reg]);
    calrhs(s, s->reg[out_reg], s->reg[in_reg]);
}

static void swapreg(orc_sim *s, int a, int b) {
    for (int f = 0; f < NF; ++f) { double *t = s->reg[a][f]; s->reg[a][f] = s->reg[b][f]; s->reg[b][f] = t; }
}

/*
 * x ghosts of a slab of an x-decomposed solve (the reference's CartGrid
 * halo exchange, nuosc_boundary.cpp:64-208, for a split in x): the callback
 * fills the x-ghost planes of register `reg` (its z ghosts are already
 * filled, z first as in nuosc_boundary.cpp:4-52) before the calRHS of stage
 * `stage`.  NULL: periodic in x inside the register.
 */
typedef void (*orc_halo_cb)(int stage, int reg, void *user);

static void ghost_fill(orc_sim *s, int reg, int stage, orc_halo_cb cb, void *user) {
    if (!cb) {
        periodic_boundary(s, s->reg[reg]);
        return;
    }
    boundary_z(s, s->reg[reg]);
    cb(stage, reg, user);
}

static void step_rk4_impl(orc_sim *s, int nsteps, orc_halo_cb cb, void *user) {
    enum { STAT = 0, RHS = 1, PRE = 2, COR = 3 };
    const double dt = s->dt;
    for (int n = 0; n < nsteps; ++n) {
        ghost_fill(s, STAT, 0, cb, user);
        calrhs(s, s->reg[RHS], s->reg[STAT]);
        vec1(s, s->reg[PRE], s->reg[STAT], 0.5 * dt, s->reg[RHS]);

        ghost_fill(s, PRE, 1, cb, user);
        calrhs(s, s->reg[COR], s->reg[PRE]);
        vec1(s, s->reg[RHS], s->reg[RHS], 2.0, s->reg[COR]);
        vec1(s, s->reg[COR], s->reg[STAT], 0.5 * dt, s->reg[COR]);
        swapreg(s, PRE, COR);

        ghost_fill(s, PRE, 2, cb, user);
        calrhs(s, s->reg[COR], s->reg[PRE]);
        vec1(s, s->reg[RHS], s->reg[RHS], 2.0, s->reg[COR]);
        vec1(s, s->reg[COR], s->reg[STAT], dt, s->reg[COR]);
        swapreg(s, PRE, COR);

        ghost_fill(s, PRE, 3, cb, user);
        calrhs(s, s->reg[COR], s->reg[PRE]);
        vec2(s, s->reg[PRE], s->reg[STAT], 1.0 / 6.0 * dt, s->reg[COR], s->reg[RHS]);
        swapreg(s, PRE, STAT);
        s->phy_time += dt;
    }
}

/* Classic RK4 exactly as step_rk4 (nuosc_class.cpp:374-427). */
void orc_step_rk4(orc_sim *s, int nsteps) { step_rk4_impl(s, nsteps, NULL, NULL); }

/* The same for one x-slab: x ghosts from the halo-exchange callback. */
void orc_step_rk4_slab(orc_sim *s, int nsteps, orc_halo_cb cb, void *user) { step_rk4_impl(s, nsteps, cb, user); }

/* Ghosted array of field f of register reg ((nx+2gx)(nz+2gz)nv doubles, CartGrid::idx order). */
double *orc_field(orc_sim *s, int reg, int f) { return s->reg[reg][f]; }

/* Global x index of local plane 0 (an x-slab): the seeded draws use it. */
void orc_set_xoff(orc_sim *s, int xoff) { s->xoff = xoff; }

/*
 * Diagnostics of analysis() (nuosc_ana.cpp:3-137), summed in (x,z,v) order.
 * out: [phy_time, maxdP, surv, survb, avgP, avgPb, aM0, Lex, ELNe]
 * (the analysis.dat column order, nuosc_ana.cpp:126-129).
 */
void orc_analysis(const orc_sim *s, double *out) {
    double maxdP = 0, avgP = 0, avgPb = 0, surv = 0, survb = 0, nor = 0, norb = 0, aM01 = 0, aM02 = 0, aM03 = 0;
    double *const *F = s->reg[0];
    for (int i = 0; i < s->nx; ++i)
        for (int j = 0; j < s->nz; ++j)
            for (int v = 0; v < s->nv; ++v) {
                long k = gidx(s, i, j, v);
                double G = s->G0[v], Gb = s->G0b[v], w = s->vw[v];
                double iG = 1.0 / G, iGb = 1.0 / Gb;
                double P1 = 2.0 * F[2][k] * iG, P2 = -2.0 * F[3][k] * iG, P3 = (F[0][k] - F[1][k]) * iG;
                double P1b = 2.0 * F[6][k] * iGb, P2b = 2.0 * F[7][k] * iGb, P3b = (F[4][k] - F[5][k]) * iGb;
                double dP = fabs(1.0 - sqrt(P1 * P1 + P2 * P2 + P3 * P3));
                double dPb = fabs(1.0 - sqrt(P1b * P1b + P2b * P2b + P3b * P3b));
                double m = dP > dPb ? dP : dPb;
                if (m > maxdP) maxdP = m;
                surv += w * F[0][k];
                survb += w * F[4][k];
                avgP += w * G * dP;
                avgPb += w * Gb * dPb;
                aM01 += w * (F[2][k] - F[6][k]);
                aM02 += w * (-F[3][k] - F[7][k]);
                aM03 += w * 0.5 * (F[0][k] - F[1][k] - F[4][k] + F[5][k]);
                nor += w * G;
                norb += w * Gb;
            }
    surv /= nor;
    survb /= norb;
    avgP /= nor;
    avgPb /= norb;
    out[0] = s->phy_time;
    out[1] = maxdP;
    out[2] = surv;
    out[3] = survb;
    out[4] = avgP;
    out[5] = avgPb;
    out[6] = sqrt(aM01 * aM01 + aM02 * aM02 + aM03 * aM03) * s->ds_L;
    out[7] = aM03 * s->ds_L;
    out[8] = fabs(s->n_nue0[0] * (1.0 - surv) - s->n_nue0[1] * (1.0 - survb)) / (s->n_nue0[0] + s->n_nue0[1]);
}
