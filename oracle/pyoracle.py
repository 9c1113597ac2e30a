"""ctypes bindings for the checkers (TEST INFRASTRUCTURE ONLY).

`Oracle` drives liboracle.so, the C restatement of nuosc's RK4 step in
oracle/nuosc_oracle.c.  `RefSim` drives oracle/_ref/libnuosc_ref_ko{6,4}.so,
the reference's own CPU sources compiled by oracle/Makefile.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.

Both expose the same small surface:
    create(...), fill_init(...), get_state(reg) -> (8, nx, nz, nv) float64,
    set_state(reg, arr), calrhs(), step(n), analysis() -> 9 floats,
    velocities() -> (vx, vy, vz, vw, G0, G0b), info
Register ids follow NuOsc (nuosc_class.h:108): 0 v_stat, 1 v_rhs, 2 v_pre, 3 v_cor.
"""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = {6: os.path.join(HERE, "_ref", "libnuosc_ref_ko6.so"),
          4: os.path.join(HERE, "_ref", "libnuosc_ref_ko4.so")}

_D = C.c_double
_I = C.c_int
_P = C.c_void_p
_DP = C.POINTER(C.c_double)

# callback of orc_step_rk4_slab: (stage, register) -> fill the x-ghost planes
HALO_CB = C.CFUNCTYPE(None, _I, _I, _P)

DIAG_NAMES = ["phy_time", "maxdP", "surv", "survb", "avgP", "avgPb", "aM0", "Lex", "ELNe"]


def build_oracle():
    """Build liboracle.so (plain gcc, a few seconds) when it is missing."""
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return ORACLE_SO


def ref_available(ko_order=6):
    return os.path.exists(REF_SO[ko_order])


def _dp(a):
    return a.ctypes.data_as(_DP)


_olib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        lib = C.CDLL(build_oracle())
        lib.orc_create.restype = _P
        lib.orc_create.argtypes = [_I, _D, _D, _D, _D, _D, _D, _D, _D, _I, _D, _D]
        lib.orc_destroy.argtypes = [_P]
        lib.orc_info.argtypes = [_P, C.POINTER(_I), _DP]
        lib.orc_velocities.argtypes = [_P] + [_DP] * 6
        lib.orc_fill_init.argtypes = [_P, _I, _D, _D, _D, _D, _D, _D, _D, C.c_uint64]
        lib.orc_set_state.argtypes = [_P, _I, _I, _DP]
        lib.orc_get_state.argtypes = [_P, _I, _I, _DP]
        lib.orc_set_g0.argtypes = [_P, _DP, _DP, _D, _D]
        lib.orc_set_time.argtypes = [_P, _D]
        lib.orc_calrhs.argtypes = [_P, _I, _I]
        lib.orc_step_rk4.argtypes = [_P, _I]
        lib.orc_analysis.argtypes = [_P, _DP]
        lib.orc_analysis.restype = None
        lib.orc_icosahedron.argtypes = [_I] + [_DP] * 4
        lib.orc_nv.restype = _I
        lib.orc_nv.argtypes = [_I]
        lib.orc_uniform.restype = _D
        lib.orc_uniform.argtypes = [C.c_uint64, _I, _I]
        lib.orc_set_noc_phases.argtypes = [_P, _I, _DP]
        lib.orc_step_rk4_slab.argtypes = [_P, _I, HALO_CB, _P]
        lib.orc_field.restype = _DP
        lib.orc_field.argtypes = [_P, _I, _I]
        lib.orc_set_xoff.argtypes = [_P, _I]
        lib.orc_adv_integrals.argtypes = [_P, _DP]
        lib.orc_adv_integrals.restype = None
        _olib = lib
    return _olib


def icosahedron(nn):
    """(vx, vy, vz, vw) of the subdivided icosahedron, restated in C."""
    lib = _oracle_lib()
    nv = lib.orc_nv(nn)
    out = [np.zeros(nv) for _ in range(4)]
    lib.orc_icosahedron(nn, *[_dp(a) for a in out])
    return tuple(out)


def uniform01(seed, i, j):
    return _oracle_lib().orc_uniform(seed, i, j)


class _Sim:
    lib = None
    h = None

    def info(self):
        ints = (_I * 4)()
        dbl = (_D * 5)()
        self._info(self.h, ints, dbl)
        return dict(nx=ints[0], nz=ints[1], nv=ints[2], ghost=ints[3], dt=dbl[0], ds_L=dbl[1],
                    phy_time=dbl[2], n_nue0=(dbl[3], dbl[4]))

    @property
    def shape(self):
        i = self.info()
        return (i["nx"], i["nz"], i["nv"])

    def velocities(self):
        nv = self.shape[2]
        out = [np.zeros(nv) for _ in range(6)]
        self._vel(self.h, *[_dp(a) for a in out])
        return tuple(out)

    def get_state(self, reg=0):
        nx, nz, nv = self.shape
        out = np.zeros((8, nx, nz, nv))
        for f in range(8):
            self._get(self.h, reg, f, _dp(out[f]))
        return out

    def set_state(self, arr, reg=0):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        for f in range(8):
            self._set(self.h, reg, f, _dp(arr[f]))

    def analysis(self):
        out = np.zeros(9)
        rc = self._ana(self.h, _dp(out))
        if rc not in (None, 0):
            raise RuntimeError("analysis failed: %r" % rc)
        return out


class Oracle(_Sim):
    """The C restatement (nuosc_oracle.c).  ko_order 6 -> 3 ghosts, 4 -> 2 ghosts."""

    def __init__(self, nn, x0, x1, z0, z1, dx, dz, cfl, ko, ko_order=6, mu=1.0, pmo=0.0):
        self.lib = lib = _oracle_lib()
        ghost = 3 if ko_order == 6 else 2
        self.h = lib.orc_create(nn, x0, x1, z0, z1, dx, dz, cfl, ko, ghost, mu, pmo)
        self._info, self._vel = lib.orc_info, lib.orc_velocities
        self._get, self._set = (lambda h, r, f, p: lib.orc_get_state(h, r, f, p)), lib.orc_set_state
        self._ana = lib.orc_analysis

    def fill_init(self, ipt=1, alpha=0.9, eps0=1e-6, sigma=1.0, lnue=0.6, lnueb=0.5, lnuex=0.0,
                  lnuebx=0.0, seed=0):
        self.lib.orc_fill_init(self.h, ipt, alpha, eps0, sigma, lnue, lnueb, lnuex, lnuebx, seed)

    def set_g0(self, G0, G0b, n0, n1):
        G0 = np.ascontiguousarray(G0, dtype=np.float64)
        G0b = np.ascontiguousarray(G0b, dtype=np.float64)
        self.lib.orc_set_g0(self.h, _dp(G0), _dp(G0b), n0, n1)

    def set_time(self, t):
        self.lib.orc_set_time(self.h, t)

    def set_xoff(self, xoff):
        """This oracle is an x-slab whose plane 0 is global plane xoff (seeded draws)."""
        self.lib.orc_set_xoff(self.h, int(xoff))

    def field(self, reg, f):
        """Ghosted array of one field of a register, a numpy view ((nx+2g)(nz+2g)nv,
        CartGrid::idx order)."""
        i = self.info()
        g = i["ghost"]
        n = (i["nx"] + 2 * g) * (i["nz"] + 2 * g) * i["nv"]
        return np.ctypeslib.as_array(self.lib.orc_field(self.h, reg, f), shape=(n,))

    def step_slab(self, n, fill_x_ghosts):
        """n RK4 steps of an x-slab: before each calRHS the z ghosts are filled
        periodically and fill_x_ghosts(stage, reg) must fill the x ghosts."""
        cb = HALO_CB(lambda stage, reg, user: fill_x_ghosts(stage, reg))
        self.lib.orc_step_rk4_slab(self.h, n, cb, None)

    def set_noc_phases(self, phi):
        """Explicit phases of the ipt = 4 initial data (None: the seeded ones)."""
        if phi is None:
            self.lib.orc_set_noc_phases(self.h, 0, None)
        else:
            phi = np.ascontiguousarray(phi, dtype=np.float64)
            self.lib.orc_set_noc_phases(self.h, len(phi), _dp(phi))

    def adv_integrals(self):
        """(I1, I2) of the advection test (nuosc_ana.cpp:58-61)."""
        out = np.zeros(2)
        self.lib.orc_adv_integrals(self.h, _dp(out))
        return out

    def calrhs(self):
        self.lib.orc_calrhs(self.h, 1, 0)

    def step(self, n=1):
        self.lib.orc_step_rk4(self.h, n)

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    __del__ = close


class RefSim(_Sim):
    """The reference's own NuOsc (oracle/_ref), driven through ref_capi.cpp."""

    _libs = {}

    def __init__(self, nn, x0, x1, z0, z1, dx, dz, cfl, ko, ko_order=6, mu=1.0, pmo=0.0, workdir=None):
        if ko_order not in RefSim._libs:
            if not ref_available(ko_order):
                raise FileNotFoundError(REF_SO[ko_order])
            lib = C.CDLL(REF_SO[ko_order])
            lib.ref_create.restype = _P
            lib.ref_create.argtypes = [_I, _D, _D, _D, _D, _D, _D, _D, _D, _I, _D, _D, C.c_char_p]
            lib.ref_destroy.argtypes = [_P]
            lib.ref_info.argtypes = [_P, C.POINTER(_I), _DP]
            lib.ref_velocities.argtypes = [_P] + [_DP] * 6
            lib.ref_fill_init.argtypes = [_P, _I, _D, _D, _D, _D, _D, _D, _D, C.c_uint64]
            lib.ref_get_state.argtypes = [_P, _I, _I, _DP]
            lib.ref_set_state.argtypes = [_P, _I, _I, _DP]
            lib.ref_calrhs.argtypes = [_P]
            lib.ref_step.argtypes = [_P, _I]
            lib.ref_analysis.argtypes = [_P, _DP]
            lib.ref_analysis.restype = _I
            lib.ref_snapshot_at_v.argtypes = [_P, C.c_char_p, _I, _I, C.POINTER(_I), _I, C.POINTER(_I), _I]
            lib.ref_snapshot_at_xv.argtypes = [_P, C.c_char_p, _I, _I, C.POINTER(_I), _I, C.POINTER(_I), _I,
                                               C.POINTER(_I), _I]
            RefSim._libs[ko_order] = lib
        self.lib = lib = RefSim._libs[ko_order]
        self._tmp = None
        if workdir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="nuosc_ref_")
            workdir = self._tmp.name
        self.workdir = workdir
        ghost = 3 if ko_order == 6 else 2
        self.h = lib.ref_create(nn, x0, x1, z0, z1, dx, dz, cfl, ko, ghost, mu, pmo, workdir.encode())
        if not self.h:
            raise RuntimeError("ref_create failed")
        self._info, self._vel = lib.ref_info, lib.ref_velocities
        self._get, self._set = lib.ref_get_state, lib.ref_set_state
        self._ana = lib.ref_analysis

    def fill_init(self, ipt=1, alpha=0.9, eps0=1e-6, sigma=1.0, lnue=0.6, lnueb=0.5, lnuex=0.0,
                  lnuebx=0.0, seed=0):
        self.lib.ref_fill_init(self.h, ipt, alpha, eps0, sigma, lnue, lnueb, lnuex, lnuebx, seed)

    def calrhs(self):
        self.lib.ref_calrhs(self.h)

    def step(self, n=1):
        self.lib.ref_step(self.h, n)

    def snapshot_at_v(self, fntpl, vidx, fields, t, every=1):
        vi = (_I * len(vidx))(*vidx)
        fi = (_I * len(fields))(*fields)
        self.lib.ref_snapshot_at_v(self.h, fntpl.encode(), every, len(vidx), vi, len(fields), fi, t)

    def snapshot_at_xv(self, fntpl, xidx, vidx, fields, t, every=1):
        xi = (_I * len(xidx))(*xidx)
        vi = (_I * len(vidx))(*vidx)
        fi = (_I * len(fields))(*fields)
        self.lib.ref_snapshot_at_xv(self.h, fntpl.encode(), every, len(xidx), xi, len(vidx), vi,
                                    len(fields), fi, t)

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None

    __del__ = close


def box(n_cells, dx):
    """Symmetric periodic box [-L, L) with n_cells cells of width dx."""
    L = n_cells * dx / 2.0
    return -L, L


def relerr(a, b):
    """Norm-wise relative error max|a-b| / max|b| (0 when both vanish)."""
    d = float(np.max(np.abs(np.asarray(a) - np.asarray(b))))
    m = float(np.max(np.abs(b)))
    return d / m if m > 0 else d
