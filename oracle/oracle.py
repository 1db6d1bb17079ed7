"""ORACLE — TEST INFRASTRUCTURE ONLY.

ctypes wrapper of liboracle.so, the CPU restatement of the reference's
RHSCAL/RHSVEL/TEMPER/CHRATE/derivatives/LINCOM path (senga_oracle.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
it, and only to check results or as the timed CPU baseline, never as the product.
Parity unpinned against outputs of the reference: it is Fortran and no
Fortran compiler exists in this build environment, and the reference ships
no tests. The oracle is pinned by known-answer tests instead
(tests/test_oracle_kat.py: constants read from the reference sources,
closed-form answers, RK order, conservation, committed fixtures).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build():
    subprocess.run(["make", "-C", HERE, "-s"], check=True)


class _Bc(C.Structure):
    _fields_ = [("xl", C.c_int), ("xr", C.c_int), ("u_in", C.c_double), ("rho_in", C.c_double),
                ("y_in", C.c_double * 18), ("p_inf", C.c_double), ("sigma", C.c_double), ("eta", C.c_double),
                ("pio", C.c_int), ("bet_local", C.c_int), ("t_in", C.c_double),
                ("t_wall", C.c_double * 2), ("nrieta", C.c_double * 6)]


class _Cfg(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("xgdlen", C.c_double), ("ygdlen", C.c_double), ("zgdlen", C.c_double),
                ("nend", C.c_int * 6), ("flmavt", C.c_int), ("tstep", C.c_double),
                ("chem_path", C.c_char_p), ("diff_path", C.c_char_p)]


_lib = None


def _get():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_create.argtypes = [C.POINTER(_Cfg)]
        lib.oracle_destroy.argtypes = [C.c_void_p]
        lib.oracle_nspec.argtypes = [C.c_void_p]
        lib.oracle_last_error.restype = C.c_char_p
        lib.oracle_set_state.argtypes = [C.c_void_p, dp, dp, ip]
        lib.oracle_get_state.argtypes = [C.c_void_p, dp, dp, ip]
        lib.oracle_step.argtypes = [C.c_void_p, C.c_int]
        lib.oracle_rhs.argtypes = [C.c_void_p, dp, dp, dp]
        lib.oracle_deriv.argtypes = [C.c_void_p, C.c_int, dp, dp]
        lib.oracle_chrate.argtypes = [C.c_void_p, dp]
        lib.oracle_flamin.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, dp, dp]
        lib.oracle_tempin.argtypes = [C.c_void_p, C.c_double, C.c_int, dp, ip, dp, C.POINTER(C.c_long)]
        lib.oracle_chem_scalar.argtypes = [C.c_void_p, C.c_char_p, dp]
        lib.oracle_filter.argtypes = [C.c_void_p, C.c_int]
        lib.oracle_set_adaptive.argtypes = [C.c_void_p, C.c_int]
        lib.oracle_set_radiation.argtypes = [C.c_void_p, C.c_char_p, C.c_double]
        lib.oracle_post.argtypes = [C.c_void_p, dp]
        lib.oracle_turbin.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, dp, dp]
        lib.oracle_ranuni.argtypes = [C.c_int, C.c_int64, dp]
        lib.oracle_set_transport.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]
        lib.oracle_set_bc.argtypes = [C.c_void_p, C.POINTER(_Bc)]
        lib.oracle_set_synth.argtypes = [C.c_void_p, C.c_double, C.c_double] + [C.c_int] * 6
        lib.oracle_tstep.argtypes = [C.c_void_p, dp, dp, C.POINTER(C.c_int)]
        lib.oracle_filter_field.argtypes = [C.c_void_p, C.c_int, dp, dp]
        lib.oracle_chem_table.argtypes = [C.c_char_p, C.c_char_p, dp, C.c_int]
        lib.oracle_substage.argtypes = [C.c_void_p, C.c_int]
        lib.oracle_set_threads.argtypes = [C.c_int]
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """CPU restatement of one rank of the reference, same interface as Box."""

    def __init__(self, shape, lengths, chem_path, diff_path, tstep, nend=(2,) * 6):
        lib = _get()
        nx, ny, nz = shape
        self.shape = (nz, ny, nx)
        cfg = _Cfg()
        cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
        cfg.xgdlen, cfg.ygdlen, cfg.zgdlen = lengths
        for i, v in enumerate(nend):
            cfg.nend[i] = v
        cfg.flmavt = 1 if diff_path else 0
        cfg.tstep = tstep
        self._chem = chem_path.encode()
        self._diff = diff_path.encode() if diff_path else None
        cfg.chem_path = self._chem
        cfg.diff_path = self._diff
        h = lib.oracle_create(C.byref(cfg))
        if not h:
            raise RuntimeError("oracle_create: " + lib.oracle_last_error().decode())
        self.h = h
        self.nspec = lib.oracle_nspec(h)
        self.nc = 5 + self.nspec

    def close(self):
        if self.h:
            _get().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _itn_shape(self):
        """ITNDEX arrays: 15 species per word, words slowest beyond one."""
        nw = (self.nspec + 14) // 15
        return self.shape if nw == 1 else (nw,) + self.shape

    def upload(self, fields, trun, itndex):
        f = np.ascontiguousarray(fields, dtype=np.float64)
        t = np.ascontiguousarray(trun, dtype=np.float64)
        it = np.ascontiguousarray(itndex, dtype=np.int32)
        assert it.shape == self._itn_shape()
        _get().oracle_set_state(self.h, _dp(f), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32)))

    def download(self):
        f = np.empty((self.nc,) + self.shape)
        t = np.empty(self.shape)
        it = np.empty(self._itn_shape(), dtype=np.int32)
        _get().oracle_get_state(self.h, _dp(f), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32)))
        return f, t, it

    def step(self, nsteps=1):
        if _get().oracle_step(self.h, nsteps) != 0:
            raise RuntimeError("oracle_step: " + _get().oracle_last_error().decode())

    def substage(self, irk):
        """One RK substage irk (1..5); BOUNTT (and ADAPTT) follow the fifth."""
        if _get().oracle_substage(self.h, int(irk)) != 0:
            raise RuntimeError("oracle_substage: " + _get().oracle_last_error().decode())

    @staticmethod
    def set_threads(n):
        _get().oracle_set_threads(int(n))

    def rhs(self):
        r = np.empty((self.nc,) + self.shape)
        t = np.empty(self.shape)
        p = np.empty(self.shape)
        if _get().oracle_rhs(self.h, _dp(r), _dp(t), _dp(p)) != 0:
            raise RuntimeError("oracle_rhs: " + _get().oracle_last_error().decode())
        return r, t, p

    def chrate(self):
        r = np.empty((self.nspec,) + self.shape)
        if _get().oracle_chrate(self.h, _dp(r)) != 0:
            raise RuntimeError("oracle_chrate: " + _get().oracle_last_error().decode())
        return r

    def flamin(self, trin, prin, drin, urin, v=None, w=None):
        """FLAMIN's planar flame and INDATA's conversion to the conserved state."""
        va = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        if _get().oracle_flamin(self.h, float(trin), float(prin), float(drin), float(urin),
                                None if va is None else _dp(va), None if wa is None else _dp(wa)) != 0:
            raise RuntimeError("oracle_flamin: " + _get().oracle_last_error().decode())

    def tempin(self, trin, maxbis=200):
        """TEMPIN on the state set last (its U register): T, ITNDEX, p and
        (bracket failures, bisection-limit failures)."""
        t = np.empty(self.shape)
        it = np.empty(self._itn_shape(), dtype=np.int32)
        p = np.empty(self.shape)
        nf = (C.c_long * 2)()
        _get().oracle_tempin(self.h, float(trin), int(maxbis), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32)), _dp(p),
                             nf)
        return t, it, p, (nf[0], nf[1])

    def deriv(self, kind, f):
        a = np.ascontiguousarray(f, dtype=np.float64)
        out = np.empty_like(a)
        if _get().oracle_deriv(self.h, kind, _dp(a), _dp(out)) != 0:
            raise RuntimeError("oracle_deriv: " + _get().oracle_last_error().decode())
        return out

    def set_bc(self, bc):
        """NSCBC x faces: bc = dict(xl, xr in {0, 11, 12, 13, 14, 21, 31, 32}, u_in, rho_in,
        y_in, p_inf, sigma, eta, pio=0, bet_local=0, t_in (I2; the I4 target),
        t_wall (W2: x-left, x-right), nrieta (I4: six relaxation
        coefficients)); 14 (I4) on the x-left face only; 31 is the W1 wall,
        32 the W2 wall."""
        b = _Bc()
        b.xl, b.xr = bc.get("xl", 0), bc.get("xr", 0)
        b.u_in, b.rho_in = bc.get("u_in", 0.0), bc.get("rho_in", 0.0)
        for i, v in enumerate(bc.get("y_in", ())):
            b.y_in[i] = v
        b.p_inf, b.sigma, b.eta = bc.get("p_inf", 0.0), bc.get("sigma", 0.0), bc.get("eta", 0.0)
        b.pio, b.bet_local = bc.get("pio", 0), bc.get("bet_local", 0)
        b.t_in = bc.get("t_in", 0.0)
        b.t_wall[0], b.t_wall[1] = bc.get("t_wall", (0.0, 0.0))
        for i, v in enumerate(bc.get("nrieta", ())):
            b.nrieta[i] = v
        if _get().oracle_set_bc(self.h, C.byref(b)) != 0:
            raise RuntimeError("oracle_set_bc: " + _get().oracle_last_error().decode())

    def set_synth(self, urms, coflow=0.0, lnx=30, lny=30, lnz=30, nfy=60, nfz=60, itime0=1):
        """Synthetic turbulent inflow velocity on the I3 x-left face (inflow.f,
        BCUTXL NXLPRM(1) = 4); itime0: the step number of the next step."""
        if _get().oracle_set_synth(self.h, float(urms), float(coflow), int(lnx), int(lny), int(lnz), int(nfy),
                                   int(nfz), int(itime0)) != 0:
            raise RuntimeError("oracle_set_synth: " + _get().oracle_last_error().decode())

    def set_radiation(self, radn_path, trefrn=300.0):
        """RADCAL on (radn.dat path, TREFRN) or off (radn_path None)."""
        p = None if radn_path is None else str(radn_path).encode()
        if _get().oracle_set_radiation(self.h, p, float(trefrn)) != 0:
            raise RuntimeError("oracle_set_radiation: " + _get().oracle_last_error().decode())

    def post(self):
        """Post-processing record fields (7 + 2 nspec, nz, ny, nx)."""
        out = np.empty((7 + 2 * self.nspec,) + self.shape)
        _get().oracle_post(self.h, _dp(out))
        return out

    def set_transport(self, mixw=False, mixp=False, soret=False, dufour=False, wmltdr=5.0):
        """cont.dat transport switches (molar mass, pressure, Soret, Dufour;
        light-species molar-mass limit)."""
        if _get().oracle_set_transport(self.h, int(mixw), int(mixp), int(soret), int(dufour), float(wmltdr)) != 0:
            raise RuntimeError("oracle_set_transport: " + _get().oracle_last_error().decode())

    def set_adaptive(self, on=True):
        _get().oracle_set_adaptive(self.h, 1 if on else 0)

    def tstep(self):
        t, e, i = C.c_double(), C.c_double(), C.c_int()
        _get().oracle_tstep(self.h, C.byref(t), C.byref(e), C.byref(i))
        return t.value, e.value, i.value

    def filter(self, mode=0):
        """FLTREM on the registers; mode bit 0 flips TWFACT, bit 1 also filters S."""
        if _get().oracle_filter(self.h, mode) != 0:
            raise RuntimeError("oracle_filter: " + _get().oracle_last_error().decode())

    def filter_field(self, f, mode=0):
        a = np.ascontiguousarray(f, dtype=np.float64)
        out = np.empty_like(a)
        if _get().oracle_filter_field(self.h, mode, _dp(a), _dp(out)) != 0:
            raise RuntimeError("oracle_filter_field: " + _get().oracle_last_error().decode())
        return out

    def scalar(self, name):
        v = C.c_double()
        _get().oracle_chem_scalar(self.h, name.encode(), C.byref(v))
        return v.value


class OracleChem:
    """chem.dat tables read by the oracle's own CHEMIN restatement, with the
    table(name) / nspec interface of the device library's Chem; for callers
    that must not load the device library (the CPU reference arm)."""

    NSPCMX, NSTPMX = 18, 68  # the oracle's table dimensions (oracle_tables.hpp)
    _SHAPES = {"ntint": (NSPCMX,), "rgspec": (NSPCMX,), "wmolar": (NSPCMX,), "ncpoly": (NSPCMX, 2),
               "ncenth": (NSPCMX, 2), "tinthi": (NSPCMX, 2), "tintlo": (NSPCMX, 2), "amasch": (NSPCMX, 2, 7),
               "amascp": (NSPCMX, 2, 7), "ntroe": (1,), "nsrif": (1,), "nlind": (1,), "mtlist": (NSTPMX,),
               "mslist": (NSTPMX,), "mllist": (NSTPMX,), "rctroe": (10, 12), "rcsrif": (10, 8), "rclind": (10, 4)}
    _INT = ("ntint", "ncpoly", "ncenth", "ntroe", "nsrif", "nlind", "mtlist", "mslist", "mllist")

    def __init__(self, path):
        self.path = path
        self._cache = {}
        self.nspec = int(self._read("nspec", (1,))[0])

    def _read(self, name, shape):
        out = np.empty(int(np.prod(shape)))
        cnt = _get().oracle_chem_table(self.path.encode(), name.encode(), _dp(out), out.size)
        if cnt < 0:
            raise RuntimeError("oracle_chem_table: " + _get().oracle_last_error().decode())
        return out.reshape(shape)

    def table(self, name):
        if name not in self._cache:
            a = self._read(name, self._SHAPES[name])
            self._cache[name] = a.astype(np.int32) if name in self._INT else a
        return self._cache[name]


def turbin(shape, inseed, const0, ck0):
    """TURBIN's velocity field for an (nx, ny, nz) box: (uvw (3, nz, ny, nx),
    imaginary parts left by the transform)."""
    nx, ny, nz = shape
    uvw = np.empty((3, nz, ny, nx))
    im = np.empty((3, nz, ny, nx))
    _get().oracle_turbin(nx, ny, nz, int(inseed), float(const0), float(ck0), _dp(uvw), _dp(im))
    return uvw, im


def ranuni(iseed, n):
    """The first n draws of RANUNI after RANINI(iseed)."""
    out = np.empty(n)
    _get().oracle_ranuni(int(iseed), int(n), _dp(out))
    return out

