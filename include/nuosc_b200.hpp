// nuosc_b200.hpp -- header-only C++ facade with the reference's NuOsc surface.
//
// A caller written against the reference's class NuOsc (nuosc_class.h:99-191)
// switches by including this header instead of nuosc_class.h, using
// nuosc_b200::NuOsc, and linking libnuosc_b200.so.  Constructor arguments,
// method names and their meaning are the reference's; the state lives on the
// GPU, so the public FieldVar pointers (v_stat->ee[...]) become get_field /
// set_field calls that copy one field in the reference's ghosted layout (or
// compactly), and errors surface as nuosc_b200::Error exceptions instead of
// asserts and exit() calls.
#pragma once

#include "nuosc_b200.h"

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace nuosc_b200 {

class Error : public std::runtime_error {
   public:
    Error(int code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

   private:
    int code_;
};

inline void check(int rc) {
    if (rc != NUOSC_OK) throw Error(rc, std::string("nuosc: ") + nuosc_last_error());
}

class NuOsc {
   public:
    // NuOsc(px, pz, nv, nphi, gx, gz, x0, x1, z0, z1, dx, dz, CFL, ko) (nuosc_class.cpp:454)
    NuOsc(int px, int pz, int nv, int nphi, int gx, int gz, double x0, double x1, double z0, double z1, double dx,
          double dz, double CFL, double ko, int precision = NUOSC_FP64, int device = 0) {
        nuosc_params p{};
        p.px = px;
        p.pz = pz;
        p.nv = nv;
        p.nphi = nphi;
        p.gx = gx;
        p.gz = gz;
        p.x0 = x0;
        p.x1 = x1;
        p.z0 = z0;
        p.z1 = z1;
        p.dx = dx;
        p.dz = dz;
        p.cfl = CFL;
        p.ko = ko;
        p.precision = precision;
        p.device = device;
        check(nuosc_create(&p, &h_));
        check(nuosc_get_geometry(h_, &g_));
        vx_.resize(g_.nv);
        vy_.resize(g_.nv);
        vz_.resize(g_.nv);
        vw_.resize(g_.nv);
        check(nuosc_get_velocities(h_, vx_.data(), vy_.data(), vz_.data(), vw_.data()));
    }
    ~NuOsc() { nuosc_destroy(h_); }
    NuOsc(const NuOsc &) = delete;
    NuOsc &operator=(const NuOsc &) = delete;

    // settings (nuosc_class.h:148-159)
    void set_mu(double mu) { check(nuosc_set_mu(h_, mu)); }
    void set_pmo(double pmo) { check(nuosc_set_pmo(h_, pmo)); }
    void set_renorm(bool renorm) { check(nuosc_set_renorm(h_, renorm ? 1 : 0)); }

    // geometry (CartGrid members)
    int nx() const { return g_.nx; }
    int nz() const { return g_.nz; }
    int get_nv() const { return g_.nv; }
    unsigned long get_lpts() const { return (unsigned long)(g_.nx + 2 * g_.gx) * (g_.nz + 2 * g_.gz) * g_.nv; }
    double dt() const { return g_.dt; }
    double ds_L() const { return g_.ds_L; }
    double phy_time() const {
        nuosc_geometry g;
        check(nuosc_get_geometry(h_, &g));
        return g.phy_time;
    }
    const std::vector<double> &vx() const { return vx_; }
    const std::vector<double> &vy() const { return vy_; }
    const std::vector<double> &vz() const { return vz_; }
    const std::vector<double> &vw() const { return vw_; }
    nuosc_handle *handle() { return h_; }

    // nuosc_init.cpp:17-137
    void fillInitValue(int ipt, double alpha, double eps0, double sigma, double lnue, double lnueb, double lnuex,
                       double lnuebx, uint64_t seed = 0) {
        check(nuosc_fill_init(h_, ipt, alpha, eps0, sigma, lnue, lnueb, lnuex, lnuebx, seed));
    }
    // the advection tests (nuosc_init.cpp:162-236), ipt 10 / 20 / 30 of nuosc_fill_init
    void fillInitAdvtest(double eps0, double sigma) { check(nuosc_fill_init(h_, 10, 0, eps0, sigma, 1, 1, 0, 0, 0)); }
    void fillInitSquare(double eps0, double sigma) { check(nuosc_fill_init(h_, 20, 0, eps0, sigma, 1, 1, 0, 0, 0)); }
    void fillInitTriangle(double eps0, double sigma) { check(nuosc_fill_init(h_, 30, 0, eps0, sigma, 1, 1, 0, 0, 0)); }

    // the hot path
    void updatePeriodicBoundary(int reg = NUOSC_REG_STAT) { check(nuosc_update_periodic_boundary(h_, reg)); }
    void calRHS(int out = NUOSC_REG_RHS, int in = NUOSC_REG_STAT) { check(nuosc_calrhs(h_, out, in)); }
    void vectorize(int dst, int src1, double a, int src2) { check(nuosc_vectorize(h_, dst, src1, a, src2)); }
    void vectorize(int dst, int src1, double a, int src2, int src3) {
        check(nuosc_vectorize2(h_, dst, src1, a, src2, src3));
    }
    void step_rk4(int nsteps = 1) { check(nuosc_step_rk4(h_, nsteps)); }

    // analysis(): returns the record; like the reference it prints the
    // "T= ..." line when print is set and appends to the analysis file when
    // one is open (nuosc_ana.cpp:119-129)
    // With adv_test the printed line is the advection test's (the reference
    // built with ADV_TEST, nuosc_ana.cpp:120-121): the integrals I1, I2.
    nuosc_diag analysis(bool print = false, bool adv_test = false) {
        nuosc_diag d{};
        check(nuosc_analysis(h_, &d));
        if (print && adv_test)
            printf("T= %15f  I1= %5.4e I2= %5.4e\n", d.phy_time, d.I1, d.I2);
        else if (print)
            printf("T= %15f  |dP|max= %5.4e surb= %5.4e %5.4e conP= %5.4e %5.4e |M0|= %5.4e ELNe= %g Lex= %g\n",
                   d.phy_time, d.maxdP, d.surv, d.survb, d.avgP, d.avgPb, d.aM0, d.ELNe, d.Lex);
        return d;
    }
    void open_analysis_file(const char *path = "analysis.dat") { check(nuosc_open_analysis_file(h_, path)); }
    void save_checkpoint(const char *path) { check(nuosc_save_checkpoint(h_, path)); }
    void load_checkpoint(const char *path) { check(nuosc_load_checkpoint(h_, path)); }

    // snapshots (nuosc_snapshot.cpp:13-122); fields are NUOSC_* ids
    void addSnapShotAtV(const std::vector<int> &fields, const char *fntpl, int dumpstep,
                        const std::vector<int> &vidx) {
        check(nuosc_add_snapshot_at_v(h_, fields.data(), (int)fields.size(), fntpl, dumpstep, vidx.data(),
                                      (int)vidx.size()));
    }
    void addSnapShotAtXV(const std::vector<int> &fields, const char *fntpl, int dumpstep,
                         const std::vector<int> &xidx, const std::vector<int> &vidx) {
        check(nuosc_add_snapshot_at_xv(h_, fields.data(), (int)fields.size(), fntpl, dumpstep, xidx.data(),
                                       (int)xidx.size(), vidx.data(), (int)vidx.size()));
    }
    void checkSnapShot(int t = 0) { check(nuosc_check_snapshot(h_, t)); }

    // FieldVar access: one field of one register, reference ghosted layout by default
    std::vector<double> get_field(int field, int reg = NUOSC_REG_STAT, int layout = NUOSC_LAYOUT_GHOSTED) {
        std::vector<double> out(layout == NUOSC_LAYOUT_GHOSTED ? get_lpts() : (size_t)g_.nx * g_.nz * g_.nv, 0.0);
        check(nuosc_get_state(h_, reg, field, out.data(), layout));
        return out;
    }
    void set_field(int field, const std::vector<double> &in, int reg = NUOSC_REG_STAT,
                   int layout = NUOSC_LAYOUT_GHOSTED) {
        check(nuosc_set_state(h_, reg, field, in.data(), layout));
    }

   private:
    nuosc_handle *h_ = nullptr;
    nuosc_geometry g_{};
    std::vector<double> vx_, vy_, vz_, vw_;
};

}  // namespace nuosc_b200
