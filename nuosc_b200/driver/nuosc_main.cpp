// nuosc_main.cpp -- command-line driver with the reference's interface (nuosc.cpp).
//
// Same flags, defaults and loop as the reference's main (nuosc.cpp:17-261):
// construct the solver, fill the initial data, analysis at t = 0, then
// END_STEP RK4 steps with analysis every ANA_EVERY steps and snapshot dumps
// every DUMP_EVERY steps, printing the wall time per step in the reference's
// "ns/step-grid" form and the closing [Summ] line.  The solve runs on one GPU
// through the C ABI (nuosc_b200.hpp).  Differences: --np must be 1 1 (one
// GPU per solve); --ipt 1 and --ipt 4 draw the perturbation from --seed
// instead of rand() (ipt 4 for every x, not only the x = 0 column); --ipt
// 10/20/30 run the advection tests, which the reference selects only when
// built with ADV_TEST (nuosc.cpp:155-158), and print I1, I2; extra flags
// --precision (0 FP64, 1 FP32), --seed and --device.
#include "../../include/nuosc_b200.hpp"

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <limits>

int main(int argc, char *argv[]) {
    int px = 1, pz = 1;
    double dz = 0.1, dx = 0.1;
    double x0 = -1, x1 = 1;
    double z0 = -10, z1 = 10;
    int nv_in = 33, nphi = 32;
    double cfl = 0.4, ko = 0.0;
    double mu = 1.0, pmo = 1.0;
    bool renorm = false;
    double alpha = 0.9, lnue = 0.6, lnueb = 0.53;
    double lnuex = std::numeric_limits<double>::max(), lnuebx = std::numeric_limits<double>::max();
    int ipt = 0;
    double eps0 = 0.1, sigma = 100.0;
    int ANAL_EVERY = 5, END_STEP = 5, DUMP_EVERY = 99999999;
    int gz = 3, gx = 3;  // 6th-difference KO; --gz 2 selects the 4th-difference form
    int precision = NUOSC_FP64, device = 0;
    unsigned long long seed = 0;

    auto need = [&](int t) {
        if (t + 1 >= argc) {
            printf("Missing value for %s\n", argv[t]);
            exit(1);
        }
    };
    for (int t = 1; t < argc; t++) {
        const char *a = argv[t];
        if (!strcmp(a, "--dz")) { need(t); dz = atof(argv[++t]); dx = dz; }
        else if (!strcmp(a, "--dx")) { need(t); dx = atof(argv[++t]); }
        else if (!strcmp(a, "--zmax")) { need(t); z1 = atof(argv[++t]); z0 = -z1; x1 = z1; x0 = z0; }
        else if (!strcmp(a, "--xmax")) { need(t); x1 = atof(argv[++t]); x0 = -x1; }
        else if (!strcmp(a, "--gz")) { need(t); gz = atoi(argv[++t]); gx = gz; }
        else if (!strcmp(a, "--cfl")) { need(t); cfl = atof(argv[++t]); }
        else if (!strcmp(a, "--nv")) { need(t); nv_in = atoi(argv[++t]); }
        else if (!strcmp(a, "--nphi")) { need(t); nphi = atoi(argv[++t]); }
        else if (!strcmp(a, "--ko")) { need(t); ko = atof(argv[++t]); }
        else if (!strcmp(a, "--mu")) { need(t); mu = atof(argv[++t]); }
        else if (!strcmp(a, "--pmo")) { need(t); pmo = atof(argv[++t]); }
        else if (!strcmp(a, "--renorm")) { need(t); renorm = atoi(argv[++t]) != 0; }
        else if (!strcmp(a, "--ANA_EVERY")) { need(t); ANAL_EVERY = atoi(argv[++t]); }
        else if (!strcmp(a, "--DUMP_EVERY")) { need(t); DUMP_EVERY = atoi(argv[++t]); }
        else if (!strcmp(a, "--END_STEP")) { need(t); END_STEP = atoi(argv[++t]); }
        else if (!strcmp(a, "--ANA_EVERY_T")) { need(t); ANAL_EVERY = int(atof(argv[++t]) / (cfl * dz) + 0.5); }
        else if (!strcmp(a, "--DUMP_EVERY_T")) { need(t); DUMP_EVERY = int(atof(argv[++t]) / (cfl * dz) + 0.5); }
        else if (!strcmp(a, "--END_STEP_T")) { need(t); END_STEP = int(atof(argv[++t]) / (cfl * dz) + 0.5); }
        else if (!strcmp(a, "--lnue")) { need(t); lnue = atof(argv[++t]); }
        else if (!strcmp(a, "--lnueb")) { need(t); lnueb = atof(argv[++t]); }
        else if (!strcmp(a, "--lnuex")) { need(t); lnuex = atof(argv[++t]); }
        else if (!strcmp(a, "--lnuebx")) { need(t); lnuebx = atof(argv[++t]); }
        else if (!strcmp(a, "--sigma")) { need(t); sigma = atof(argv[++t]); }
        else if (!strcmp(a, "--eps0")) { need(t); eps0 = atof(argv[++t]); }
        else if (!strcmp(a, "--alpha")) { need(t); alpha = atof(argv[++t]); }
        else if (!strcmp(a, "--ipt")) { need(t); ipt = atoi(argv[++t]); }
        else if (!strcmp(a, "--np")) { need(t + 1); px = atoi(argv[++t]); pz = atoi(argv[++t]); }
        else if (!strcmp(a, "--precision")) { need(t); precision = atoi(argv[++t]); }
        else if (!strcmp(a, "--seed")) { need(t); seed = strtoull(argv[++t], nullptr, 10); }
        else if (!strcmp(a, "--device")) { need(t); device = atoi(argv[++t]); }
        else {
            printf("Unreconganized parameters %s!\n", a);
            return 0;
        }
    }

    try {
        nuosc_b200::NuOsc state(px, pz, nv_in, nphi, gx, gz, x0, x1, z0, z1, dx, dz, cfl, ko, precision, device);
        const unsigned long lpts = state.get_lpts();
        printf("\nNuOsc2D on 1 GPU (%s state)\n", precision == NUOSC_FP64 ? "FP64" : "FP32");
        printf("   Domain:  v: nv = %5d  on S2.\n", state.get_nv());
        printf("            x:( %12f %12f )  dx = %g\n", x0, x1, dx);
        printf("            z:( %12f %12f )  dz = %g\n", z0, z1, dz);
        printf("   dt = %g     CFL = %g\n", state.dt(), cfl);
        printf("   Dissipation: %s KO w/ eps = %g\n", gx == 3 ? "6th-difference" : "4th-difference", ko);
        state.set_mu(mu);
        state.set_pmo(pmo);
        state.set_renorm(renorm);
        printf("   Setting mu = %f\n   Setting pmo = %f\n   Setting renorm = %d\n", mu, pmo, (int)renorm);
        state.open_analysis_file("analysis.dat");
        // ipt 10/20/30: the advection tests, which the reference's driver selects
        // when built with ADV_TEST (nuosc.cpp:155-158); their analysis line
        // prints the integrals I1, I2
        const bool adv = ipt == 10 || ipt == 20 || ipt == 30;
        if (ipt == 10) state.fillInitAdvtest(eps0, sigma);
        else if (ipt == 20) state.fillInitSquare(eps0, sigma);
        else if (ipt == 30) state.fillInitTriangle(eps0, sigma);
        else state.fillInitValue(ipt, alpha, eps0, sigma, lnue, lnueb, lnuex, lnuebx, seed);
        state.analysis(true, adv);

        if (DUMP_EVERY <= END_STEP) {
            std::vector<int> vslice;
            for (int v = 0; v < state.get_nv(); v += (state.get_nv() > 16 ? state.get_nv() / 16 : 1))
                vslice.push_back(v);
            state.addSnapShotAtV({NUOSC_P3}, "P3_%06d.bin", DUMP_EVERY, vslice);
            state.checkSnapShot(0);
        }

        const int cooltime = 3;
        auto t1 = std::chrono::high_resolution_clock::now();
        double stepms = 0;
        for (int t = 1; t <= END_STEP; t++) {
            if (t == cooltime) {  // start the clock at step 3 as the reference does (nuosc.cpp:204-211)
                nuosc_synchronize(state.handle());
                t1 = std::chrono::high_resolution_clock::now();
            }
            state.step_rk4(1);
            if (t % ANAL_EVERY == 0) state.analysis(true, adv);
            if (t % DUMP_EVERY == 0) state.checkSnapShot(t);
            if (t == 5 || t == 10 || t == 100 || t == 1000 || t == END_STEP) {
                nuosc_synchronize(state.handle());
                stepms = std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t1)
                             .count();
                const int n = t - cooltime + 1 > 0 ? t - cooltime + 1 : 1;
                printf("%d Walltime: %.3f s/T, %.2f ns/step-grid.\n", t, stepms / state.phy_time() / 1000,
                       stepms / n / lpts * 1e6);
            }
        }
        const int n = END_STEP - cooltime + 1 > 0 ? END_STEP - cooltime + 1 : 1;
        printf("Completed.\n");
        printf("[Summ] %d %d %d %d %d %d %f\n", 1, px, pz, state.nx(), state.nz(), state.get_nv(),
               stepms / n / lpts * 1e6);
    } catch (const nuosc_b200::Error &e) {
        fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
