"""Host-side Python interface to libsenga_gpu.so (the B200 SENGA2 RHS/RK path).

Mirrors the reference's call surfaces for this path:
  * CHEMIN / DIFFIN table set-up            -> Chem.load / Diff.load
  * the COMMON-resident state of one rank   -> Box (device-resident context)
  * RHSCAL + RHSVEL                         -> Box.rhs()
  * one substage / one RK step              -> Box.substage(irk) / Box.step(n)
  * DFBYDX..D2FDYZ(FUNCTN, FDERIV)          -> Box.dfbydx(f) ... Box.d2fdyz(f)
  * TEMPER, CHRATE                          -> Box.temper(), Box.chrate()

Arrays are numpy float64 with shape (..., nz, ny, nx) in C order, which is
the reference's Fortran (nx, ny, nz) column-major layout byte for byte.
The CUDA library is required: importing this module fails loudly when
libsenga_gpu.so is missing or cannot be loaded; there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsenga_gpu.so")
DATA = os.path.join(HERE, "data")

NSPCMX, NSTPMX, NTINMX, NCOFMX, NSSMAX, NBDYMX, NLLMAX, NDCFMX = 18, 68, 2, 7, 10, 10, 10, 4
NSPIMX = 15  # species per ITNDEX word


def itn_words(nspec):
    """32-bit ITNDEX words per grid point (base-4 digits, 15 species a word)."""
    return (nspec + NSPIMX - 1) // NSPIMX


def itn_shape(nspec, shape):
    """Host shape of an ITNDEX array: the grid's for up to 15 species, else
    (words,) + the grid's, words slowest."""
    w = itn_words(nspec)
    return tuple(shape) if w == 1 else (w,) + tuple(shape)
NOBC, NBOUND, NPERI = 0, 1, 2


def _arr(t, *dims):
    for d in reversed(dims):
        t = t * d
    return t


class ChemT(C.Structure):
    """senga_chem: COMMON/CHEMIC after CHEMIN (src/com_senga2.h:121-178)."""

    _fields_ = [
        ("nspec", C.c_int), ("nstep", C.c_int), ("nbody", C.c_int), ("ngibb", C.c_int),
        ("nlind", C.c_int), ("ntroe", C.c_int), ("nsrif", C.c_int),
        ("ntint", _arr(C.c_int, NSPCMX)),
        ("ncofcp", _arr(C.c_int, NSPCMX, NTINMX)), ("ncpoly", _arr(C.c_int, NSPCMX, NTINMX)),
        ("ncpom1", _arr(C.c_int, NSPCMX, NTINMX)), ("ncenth", _arr(C.c_int, NSPCMX, NTINMX)),
        ("ncenpy", _arr(C.c_int, NSPCMX, NTINMX)),
        ("nsslen", _arr(C.c_int, NSTPMX)), ("nrslen", _arr(C.c_int, NSTPMX)),
        ("npslen", _arr(C.c_int, NSTPMX)), ("nrclen", _arr(C.c_int, NSTPMX)),
        ("npclen", _arr(C.c_int, NSTPMX)),
        ("nsspec", _arr(C.c_int, NSTPMX, NSSMAX)), ("nrspec", _arr(C.c_int, NSTPMX, NSSMAX)),
        ("npspec", _arr(C.c_int, NSTPMX, NSSMAX)), ("nrcpec", _arr(C.c_int, NSTPMX, NSSMAX)),
        ("npcpec", _arr(C.c_int, NSTPMX, NSSMAX)),
        ("mblist", _arr(C.c_int, NSTPMX)), ("mglist", _arr(C.c_int, NSTPMX)),
        ("mllist", _arr(C.c_int, NSTPMX)), ("mtlist", _arr(C.c_int, NSTPMX)),
        ("mslist", _arr(C.c_int, NSTPMX)),
        ("prefgb", C.c_double), ("alamda", C.c_double),
        ("tintlo", _arr(C.c_double, NSPCMX, NTINMX)), ("tinthi", _arr(C.c_double, NSPCMX, NTINMX)),
        ("amolcp", _arr(C.c_double, NSPCMX, NTINMX, NCOFMX)),
        ("amolgb", _arr(C.c_double, NSPCMX, NTINMX, NCOFMX)),
        ("amascp", _arr(C.c_double, NSPCMX, NTINMX, NCOFMX)),
        ("amasct", _arr(C.c_double, NSPCMX, NTINMX, NCOFMX)),
        ("amasch", _arr(C.c_double, NSPCMX, NTINMX, NCOFMX)),
        ("amascs", _arr(C.c_double, NSPCMX, NTINMX, NCOFMX)),
        ("rparam", _arr(C.c_double, NSTPMX, 3)),
        ("rclind", _arr(C.c_double, NLLMAX, 4)), ("rctroe", _arr(C.c_double, NLLMAX, 12)),
        ("rcsrif", _arr(C.c_double, NLLMAX, 8)),
        ("diffmu", _arr(C.c_double, NSTPMX, NSSMAX)), ("diffmw", _arr(C.c_double, NSTPMX, NSSMAX)),
        ("crspec", _arr(C.c_double, NSTPMX, NSSMAX)), ("cpspec", _arr(C.c_double, NSTPMX, NSSMAX)),
        ("effy3b", _arr(C.c_double, NBDYMX, NSPCMX)),
        ("wmolar", _arr(C.c_double, NSPCMX)), ("ovwmol", _arr(C.c_double, NSPCMX)),
        ("rgspec", _arr(C.c_double, NSPCMX)), ("clewis", _arr(C.c_double, NSPCMX)),
        ("olewis", _arr(C.c_double, NSPCMX)),
    ]


class DiffT(C.Structure):
    """senga_diff: COMMON/DIFFUS after DIFFIN (src/com_senga2.h:189-214)."""

    _fields_ = [
        ("flmavt", C.c_int), ("ncodif", C.c_int), ("ncotdr", C.c_int), ("ncovis", C.c_int),
        ("ncocon", C.c_int), ("pdifgb", C.c_double), ("tdifgb", C.c_double),
        ("diffco", _arr(C.c_double, NSPCMX, NSPCMX, NDCFMX)),
        ("tdrcco", _arr(C.c_double, NSPCMX, NSPCMX, NDCFMX)),
        ("wilko1", _arr(C.c_double, NSPCMX, NSPCMX)), ("wilko2", _arr(C.c_double, NSPCMX, NSPCMX)),
        ("viscco", _arr(C.c_double, NSPCMX, NDCFMX)), ("condco", _arr(C.c_double, NSPCMX, NDCFMX)),
    ]


class ConfigT(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xgdlen", C.c_double), ("ygdlen", C.c_double), ("zgdlen", C.c_double),
        ("nend", C.c_int * 6), ("tstep", C.c_double), ("adaptive", C.c_int), ("device", C.c_int),
    ]


class SynthT(C.Structure):
    """senga_synth_inflow: synthetic turbulent inflow velocity parameters."""

    _fields_ = [("urms", C.c_double), ("coflow", C.c_double), ("lnx", C.c_int), ("lny", C.c_int),
                ("lnz", C.c_int), ("nfy", C.c_int), ("nfz", C.c_int), ("itime", C.c_int)]


class NscbcT(C.Structure):
    """senga_nscbc: x-face kinds (11 I1, 12 I2, 13 I3, 14 I4 inflow, 21 O1 outflow, 31 W1, 32 W2 wall)
    and parameters."""

    _fields_ = [("xl", C.c_int), ("xr", C.c_int), ("u_in", C.c_double), ("rho_in", C.c_double),
                ("y_in", C.c_double * NSPCMX), ("p_inf", C.c_double), ("sigma", C.c_double), ("eta", C.c_double),
                ("pio", C.c_int), ("bet_local", C.c_int), ("t_in", C.c_double),
                ("t_wall", C.c_double * 2), ("nrieta", C.c_double * 6)]


NCFRMX = 6


class RadnT(C.Structure):
    """senga_radn: Planck-mean absorption data of the radiating species."""

    _fields_ = [("nsprad", C.c_int), ("nsprid", C.c_int * NSPCMX), ("nkprad", C.c_int * NSPCMX),
                ("akprad", (C.c_double * NCFRMX) * NSPCMX), ("trefrn", C.c_double)]


class SengaError(RuntimeError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise SengaError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
    lib = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
    i32p = C.POINTER(C.c_int32)
    sig = {
        "senga_chem_load": (ip, [C.c_char_p, C.POINTER(ChemT)]),
        "senga_diff_load": (ip, [C.c_char_p, C.POINTER(ChemT), C.POINTER(DiffT)]),
        "senga_ctx_create": (ip, [C.POINTER(ConfigT), C.POINTER(ChemT), C.POINTER(DiffT), C.POINTER(vp)]),
        "senga_ctx_destroy": (ip, [vp]),
        "senga_last_error": (C.c_char_p, []),
        "senga_sync": (ip, [vp]),
        "senga_stream": (vp, [vp]),
        "senga_upload_state_host": (ip, [vp, dp, dp, i32p]),
        "senga_download_state_host": (ip, [vp, dp, dp, i32p]),
        "senga_substage": (ip, [vp, ip]),
        "senga_step": (ip, [vp, ip]),
        "senga_step_graph": (ip, [vp, ip]),
        "senga_rhs_host": (ip, [vp, dp, dp, dp]),
        "senga_get_status": (ip, [vp, C.POINTER(C.c_int)]),
        "senga_profile_step": (ip, [vp, dp, C.POINTER(C.c_int)]),
        "senga_ctx_info": (ip, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int64)]),
        "senga_ctx_species_fused": (ip, [vp, C.POINTER(C.c_int)]),
        "senga_ctx_species_mma": (ip, [vp, C.POINTER(C.c_int)]),
        "senga_fp64_peak": (ip, [ip, dp]),
        "senga_filter": (ip, [vp, ip]),
        "senga_get_tstep": (ip, [vp, dp, dp, C.POINTER(C.c_int)]),
        "senga_set_nscbc": (ip, [vp, C.POINTER(NscbcT)]),
        "senga_set_synthetic_inflow": (ip, [vp, C.POINTER(SynthT)]),
        "senga_radn_load": (ip, [C.c_char_p, C.POINTER(ChemT), C.c_double, C.POINTER(RadnT)]),
        "senga_set_radiation": (ip, [vp, C.POINTER(RadnT)]),
        "senga_set_transport": (ip, [vp, ip, ip, ip, ip, C.c_double]),
        "senga_keep_rates": (ip, [vp, ip]),
        "senga_zgroup_set_nscbc": (ip, [vp, C.POINTER(NscbcT)]),
        "senga_zgroup_create": (ip, [C.POINTER(ConfigT), C.POINTER(ChemT), C.POINTER(DiffT), ip, C.POINTER(ip),
                                     C.POINTER(vp)]),
        "senga_zgroup_upload_host": (ip, [vp, dp, dp, i32p]),
        "senga_zgroup_download_host": (ip, [vp, dp, dp, i32p]),
        "senga_zgroup_step": (ip, [vp, ip]),
        "senga_zgroup_sync": (ip, [vp]),
        "senga_zgroup_destroy": (ip, [vp]),
        "senga_turbin_host": (ip, [ip, ip, ip, ip, C.c_double, C.c_double, dp, dp]),
        "senga_upload_state_async": (ip, [vp, dp, dp, i32p]),
        "senga_download_state_async": (ip, [vp, dp, dp, i32p]),
        "senga_post_fields_host": (ip, [vp, dp]),
        "senga_post_write": (ip, [C.c_char_p, ip, ip, ip, ip, ip, dp, C.c_double]),
        "senga_post_read": (ip, [C.c_char_p, ip, ip, ip, ip, ip, dp, dp]),
        "senga_server_set_max_points": (ip, [vp, C.c_int64]),
        "senga_dump_write": (ip, [C.c_char_p, ip, ip, ip, ip, ip, ip, dp, dp]),
        "senga_dump_read": (ip, [C.c_char_p, ip, ip, C.POINTER(C.c_int), dp, C.c_int64, dp]),
        "senga_filter_field_host": (ip, [vp, ip, dp, dp]),
        "senga_deriv": (ip, [vp, ip, vp, vp]),
        "senga_deriv_host": (ip, [vp, ip, dp, dp]),
        "senga_tempin_host": (ip, [vp, C.c_double, dp, i32p, dp]),
        "senga_flamin": (ip, [vp, C.c_double, C.c_double, C.c_double, C.c_double, dp, dp]),
        "senga_temper_host": (ip, [vp, dp, dp]),
        "senga_chrate_host": (ip, [vp, dp]),
        "senga_batch_create": (ip, [ip, C.POINTER(ConfigT), C.POINTER(ChemT), C.POINTER(DiffT), ip, C.POINTER(vp)]),
        "senga_batch_destroy": (ip, [vp]),
        "senga_batch_upload_host": (ip, [vp, ip, dp, dp, i32p]),
        "senga_batch_download_host": (ip, [vp, ip, dp, dp, i32p]),
        "senga_batch_step": (ip, [vp, ip]),
        "senga_batch_autotune": (ip, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "senga_batch_form": (ip, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "senga_batch_sync": (ip, [vp]),
        "senga_batch_stream": (vp, [vp]),
        "senga_batch_status": (ip, [vp, C.POINTER(C.c_int)]),
        "senga_server_create": (ip, [C.c_size_t, C.POINTER(ChemT), C.POINTER(DiffT), ip, C.POINTER(vp)]),
        "senga_server_destroy": (ip, [vp]),
        "senga_server_submit": (ip, [vp, C.POINTER(ConfigT), dp, dp, i32p, ip, C.POINTER(C.c_int)]),
        "senga_server_tick": (ip, [vp, C.POINTER(C.c_int)]),
        "senga_server_result": (ip, [vp, ip, dp, dp, i32p, dp]),
        "senga_server_stats": (ip, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64)]),
        "senga_rhs_noalloc": (ip, [C.POINTER(ConfigT), C.POINTER(ChemT), C.POINTER(DiffT), vp, vp, vp, vp, vp,
                                   vp]),
        "senga_deriv_big": (ip, [vp, ip, vp, vp]),
        "senga_deriv_big_host": (ip, [vp, ip, dp, dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def dump_write(path, fields, etime=0.0, tstep=0.0, errold=1.0e-4, errldr=1.0e-4, formatted=False, nspcmx=None):
    """Write a restart dump in the reference's layout. fields: (5+nspec, nz,
    ny, nx) conserved state (rho, rho u, rho v, rho w, rho E, rho Y_k)."""
    f = np.ascontiguousarray(fields, dtype=np.float64)
    nc, nz, ny, nx = f.shape
    nspec = nc - 5
    sc = np.array([etime, tstep, errold, errldr], dtype=np.float64)
    _check(lib.senga_dump_write(os.fsencode(path), 1 if formatted else 0, nx, ny, nz, nspec, nspcmx or nspec,
                                _dp(f), _dp(sc)), "senga_dump_write")


def dump_read(path, formatted=False, nspcmx=None):
    """Read a restart dump; returns (fields (5+nspec, nz, ny, nx), dict of
    etime, tstep, errold, errldr). nspcmx: the writing build's NSPCMX
    (unformatted files store that many species slots; default nspec)."""
    dims = (C.c_int * 4)()
    _check(lib.senga_dump_read(os.fsencode(path), 1 if formatted else 0, nspcmx or 99, dims, None, 0, None),
           "senga_dump_read")
    nx, ny, nz, nspec = list(dims)
    f = np.empty((5 + nspec, nz, ny, nx))
    sc = np.empty(4)
    _check(lib.senga_dump_read(os.fsencode(path), 1 if formatted else 0, nspcmx or nspec, dims, _dp(f), f.size,
                               _dp(sc)), "senga_dump_read")
    return f, dict(etime=sc[0], tstep=sc[1], errold=sc[2], errldr=sc[3])


def turbin(shape, inseed=1, const0=8.51064, ck0=5.0):
    """Initial turbulence of TURBIN on the device for an (nx, ny, nz) box:
    ((3, nz, ny, nx) velocity, largest imaginary part left)."""
    nx, ny, nz = shape
    uvw = np.empty((3, nz, ny, nx))
    im = C.c_double()
    _check(lib.senga_turbin_host(nx, ny, nz, int(inseed), float(const0), float(ck0), _dp(uvw), C.byref(im)),
           "senga_turbin_host")
    return uvw, im.value


def post_name(iddump, iproc=0):
    """File name of a post-processing record: out<IDDUMP:5><IPROC:4>.res."""
    return f"out{iddump:05d}{iproc:04d}.res"


def post_write(path, post, etime=0.0, nspcmx=None):
    """Write a post-processing record; post: (7 + 2 nspec, nz, ny, nx) as
    Box.post_fields returns it."""
    a = np.ascontiguousarray(post, dtype=np.float64)
    nf, nz, ny, nx = a.shape
    nspec = (nf - 7) // 2
    _check(lib.senga_post_write(os.fsencode(path), nx, ny, nz, nspec, nspcmx or nspec, _dp(a), float(etime)),
           "senga_post_write")


def post_read(path, shape, nspec, nspcmx=None):
    """Read a post-processing record of a (nx, ny, nz) box: (post, etime)."""
    nx, ny, nz = shape
    a = np.empty((7 + 2 * nspec, nz, ny, nx))
    e = C.c_double()
    _check(lib.senga_post_read(os.fsencode(path), nx, ny, nz, nspec, nspcmx or nspec, _dp(a), C.byref(e)),
           "senga_post_read")
    return a, e.value


def fp64_peak(device=0):
    """Measured FP64 FMA throughput of the device, TFLOP/s."""
    v = C.c_double()
    _check(lib.senga_fp64_peak(device, C.byref(v)), "senga_fp64_peak")
    return v.value


def _check(rc, what):
    if rc != 0:
        msg = lib.senga_last_error()
        raise SengaError(f"{what} failed (status {rc}): {msg.decode() if msg else ''}")


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Chem:
    """Chemistry tables (CHEMIN) loaded from a chem.dat file."""

    def __init__(self, path):
        self.path = path
        self.t = ChemT()
        _check(lib.senga_chem_load(path.encode(), C.byref(self.t)), "senga_chem_load")

    @property
    def nspec(self):
        return self.t.nspec

    def table(self, name):
        return np.ctypeslib.as_array(getattr(self.t, name))


class Diff:
    """Transport tables (DIFFIN); path=None gives constant-Lewis transport."""

    def __init__(self, path, chem):
        self.path = path
        self.t = DiffT()
        _check(lib.senga_diff_load(path.encode() if path else None, C.byref(chem.t), C.byref(self.t)),
               "senga_diff_load")

    @property
    def mixture_averaged(self):
        return bool(self.t.flmavt)


def nscbc_struct(bc):
    """senga_nscbc from a dict (see Box.set_nscbc)."""
    b = NscbcT()
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
    return b


class ZGroup:
    """One box split along z into `nslabs` contexts (on `devices`, default
    all on `device`); the stencils read z halos from the neighbouring slabs
    directly. y and z periodic; x periodic, or bounded (nend) with NSCBC
    faces set by set_nscbc."""

    def __init__(self, shape, lengths, chem, diff, tstep, nslabs, devices=None, device=0, nend=(NPERI,) * 6):
        nx, ny, nz = shape
        self.shape = (nz, ny, nx)
        self.nspec = chem.nspec
        self.nc = 5 + self.nspec
        cfg = ConfigT()
        cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
        cfg.xgdlen, cfg.ygdlen, cfg.zgdlen = lengths
        for i in range(6):
            cfg.nend[i] = nend[i]
        cfg.tstep = tstep
        cfg.adaptive = 0
        cfg.device = device
        devs = (C.c_int * nslabs)(*devices) if devices is not None else None
        h = C.c_void_p()
        _check(lib.senga_zgroup_create(C.byref(cfg), C.byref(chem.t), C.byref(diff.t), nslabs, devs, C.byref(h)),
               "senga_zgroup_create")
        self.h = h

    def upload(self, fields, trun, itndex):
        f = np.ascontiguousarray(fields, dtype=np.float64)
        t = np.ascontiguousarray(trun, dtype=np.float64)
        it = np.ascontiguousarray(itndex, dtype=np.int32)
        assert f.shape == (self.nc,) + self.shape and t.shape == self.shape
        assert it.shape == itn_shape(self.nspec, self.shape)
        _check(lib.senga_zgroup_upload_host(self.h, _dp(f), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32))),
               "senga_zgroup_upload_host")

    def set_nscbc(self, bc):
        """NSCBC x faces on every slab, from a dict as Box.set_nscbc takes."""
        _check(lib.senga_zgroup_set_nscbc(self.h, C.byref(nscbc_struct(bc))), "senga_zgroup_set_nscbc")

    def step(self, nsteps=1):
        _check(lib.senga_zgroup_step(self.h, nsteps), "senga_zgroup_step")

    def sync(self):
        _check(lib.senga_zgroup_sync(self.h), "senga_zgroup_sync")

    def download(self):
        f = np.empty((self.nc,) + self.shape)
        t = np.empty(self.shape)
        it = np.empty(itn_shape(self.nspec, self.shape), dtype=np.int32)
        _check(lib.senga_zgroup_download_host(self.h, _dp(f), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32))),
               "senga_zgroup_download_host")
        return f, t, it

    def close(self):
        if getattr(self, "h", None):
            lib.senga_zgroup_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Radn:
    """Radiation data (RADCIN) from a radn.dat file and the reference
    ambient temperature TREFRN [K] of the cont.dat radiation line."""

    def __init__(self, path, chem, trefrn=300.0):
        self.path = path
        self.t = RadnT()
        _check(lib.senga_radn_load(path.encode(), C.byref(chem.t), float(trefrn), C.byref(self.t)),
               "senga_radn_load")

    @property
    def species(self):
        """1-based indices of the radiating species."""
        return [self.t.nsprid[j] for j in range(self.t.nsprad)]

    def coefficients(self, j):
        return [self.t.akprad[j][k] for k in range(self.t.nkprad[j])]


class Box:
    """One box: HBM-resident state plus the per-substage RHS/RK path."""

    def __init__(self, shape, lengths, chem, diff, tstep, nend=(NPERI,) * 6, adaptive=False, device=0):
        nx, ny, nz = shape
        self.shape = (nz, ny, nx)
        self.chem, self.diff = chem, diff
        self.nspec = chem.nspec
        self.nc = 5 + self.nspec
        cfg = ConfigT()
        cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
        cfg.xgdlen, cfg.ygdlen, cfg.zgdlen = lengths
        for i, v in enumerate(nend):
            cfg.nend[i] = v
        cfg.tstep = tstep
        cfg.adaptive = 1 if adaptive else 0
        cfg.device = device
        self.cfg = cfg
        h = C.c_void_p()
        _check(lib.senga_ctx_create(C.byref(cfg), C.byref(chem.t), C.byref(diff.t), C.byref(h)),
               "senga_ctx_create")
        self.h = h

    def close(self):
        if self.h:
            lib.senga_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state ----
    def upload(self, fields, trun, itndex):
        f = np.ascontiguousarray(fields, dtype=np.float64)
        t = np.ascontiguousarray(trun, dtype=np.float64)
        it = np.ascontiguousarray(itndex, dtype=np.int32)
        assert f.shape == (self.nc,) + self.shape and t.shape == self.shape
        assert it.shape == itn_shape(self.nspec, self.shape)
        _check(lib.senga_upload_state_host(self.h, _dp(f), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32))),
               "upload")

    def download(self, out=None):
        """State, T and ITNDEX as host arrays; out=(fields, T, itn) reuses
        caller arrays (e.g. page-locked ones, for full-speed copies)."""
        if out is None:
            f = np.empty((self.nc,) + self.shape)
            t = np.empty(self.shape)
            it = np.empty(itn_shape(self.nspec, self.shape), dtype=np.int32)
        else:
            f, t, it = out
            assert f.shape == (self.nc,) + self.shape and f.dtype == np.float64 and f.flags.c_contiguous
            assert t.shape == self.shape and t.dtype == np.float64 and t.flags.c_contiguous
            assert it.shape == itn_shape(self.nspec, self.shape) and it.dtype == np.int32 and it.flags.c_contiguous
        _check(lib.senga_download_state_host(self.h, _dp(f), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32))),
               "download")
        return f, t, it

    # ---- hot path ----
    def substage(self, irk):
        _check(lib.senga_substage(self.h, irk), "senga_substage")

    def step(self, nsteps=1, graph=False):
        _check((lib.senga_step_graph if graph else lib.senga_step)(self.h, nsteps), "senga_step")

    def sync(self):
        _check(lib.senga_sync(self.h), "senga_sync")

    def status(self):
        s = C.c_int()
        _check(lib.senga_get_status(self.h, C.byref(s)), "senga_get_status")
        return s.value

    def profile_step(self):
        """One RK step with per-kernel-family CUDA-event timing:
        ({'thermo','flow','species_a','species_b_rk'} -> ms, launches), or
        with the species kernels fused ({'thermo','flow','species'} -> ms,
        launches)."""
        ms = np.zeros(4)
        nl = C.c_int()
        _check(lib.senga_profile_step(self.h, _dp(ms), C.byref(nl)), "senga_profile_step")
        if self.species_fused():
            return {"thermo": ms[0], "flow": ms[1], "species": ms[2] + ms[3]}, nl.value
        return dict(zip(("thermo", "flow", "species_a", "species_b_rk"), ms.tolist())), nl.value

    def species_fused(self):
        """True when the species and species+RK kernels run as one launch."""
        v = C.c_int()
        _check(lib.senga_ctx_species_fused(self.h, C.byref(v)), "senga_ctx_species_fused")
        return bool(v.value)

    def species_mma(self):
        """True when the species kernel takes its x derivatives on the FP64
        tensor cores (SENGA_SPECIES_MMA=1, all-periodic boxes with extents that
        are multiples of 8)."""
        v = C.c_int()
        _check(lib.senga_ctx_species_mma(self.h, C.byref(v)), "senga_ctx_species_mma")
        return bool(v.value)

    def info(self):
        """{'mech': thermochemistry kernel id, 'device_bytes': bytes held}."""
        m = C.c_int()
        b = C.c_int64()
        _check(lib.senga_ctx_info(self.h, C.byref(m), C.byref(b)), "senga_ctx_info")
        return {"mech": m.value, "device_bytes": b.value}

    @property
    def stream(self):
        return lib.senga_stream(self.h)

    def rhs(self):
        """RHSCAL + RHSVEL of the current U register: (R(U), T, p)."""
        r = np.empty((self.nc,) + self.shape)
        t = np.empty(self.shape)
        p = np.empty(self.shape)
        _check(lib.senga_rhs_host(self.h, _dp(r), _dp(t), _dp(p)), "senga_rhs_host")
        return r, t, p

    def temper(self):
        t = np.empty(self.shape)
        p = np.empty(self.shape)
        _check(lib.senga_temper_host(self.h, _dp(t), _dp(p)), "senga_temper_host")
        return t, p

    def chrate(self):
        r = np.empty((self.nspec,) + self.shape)
        _check(lib.senga_chrate_host(self.h, _dp(r)), "senga_chrate_host")
        return r

    # ---- derivative family (FUNCTN interior array -> FDERIV) ----
    def flamin(self, trin, prin, drin, urin, v=None, w=None):
        """FLAMIN's planar flame and INDATA's conversion to the conserved
        state on the device (v, w: (nz, ny, nx) arrays or None for zero)."""
        va = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        _check(lib.senga_flamin(self.h, float(trin), float(prin), float(drin), float(urin),
                                None if va is None else _dp(va), None if wa is None else _dp(wa)), "senga_flamin")

    def tempin(self, trin):
        """TEMPIN on the uploaded conserved state: (T, ITNDEX, p) of every
        point, also left on the device for the next step."""
        t = np.empty(self.shape)
        it = np.empty(itn_shape(self.nspec, self.shape), dtype=np.int32)
        p = np.empty(self.shape)
        _check(lib.senga_tempin_host(self.h, float(trin), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32)), _dp(p)),
               "senga_tempin_host")
        return t, it, p

    def deriv(self, kind, f):
        a = np.ascontiguousarray(f, dtype=np.float64)
        assert a.shape == self.shape
        out = np.empty_like(a)
        _check(lib.senga_deriv_host(self.h, kind, _dp(a), _dp(out)), "senga_deriv_host")
        return out

    def deriv_big(self, kind, f_big):
        """The operator on a halo-extended array (5 points per side, shape
        (nz+10, ny+10, nx+10)); returns the interior result."""
        a = np.ascontiguousarray(f_big, dtype=np.float64)
        assert a.shape == tuple(m + 10 for m in self.shape)
        out = np.empty(self.shape)
        _check(lib.senga_deriv_big_host(self.h, kind, _dp(a), _dp(out)), "senga_deriv_big_host")
        return out

    def set_nscbc(self, bc):
        """NSCBC x faces from a dict (xl, xr in {0, 12, 13, 21, 31}, u_in, rho_in,
        y_in, p_inf, sigma, eta, pio, bet_local, t_in, t_wall, nrieta); 11 I1
        inflow, 12 I2 inflow, 13 I3 inflow, 14 I4 inflow (x-left; nrieta:
        its six relaxation coefficients), 21 O1 outflow, 31 W1 adiabatic
        no-slip wall, 32 W2 isothermal no-slip wall (t_wall: x-left, x-right
        temperatures)."""
        _check(lib.senga_set_nscbc(self.h, C.byref(nscbc_struct(bc))), "senga_set_nscbc")

    def set_synthetic_inflow(self, urms, coflow=0.0, lnx=30, lny=30, lnz=30, nfy=60, nfz=60, itime=1):
        """Synthetic turbulent inflow velocity on the I3 x-left face (the
        reference's digital filter, BCUTXL NXLPRM(1) = 4); itime: the step
        number of the next step."""
        p = SynthT(float(urms), float(coflow), int(lnx), int(lny), int(lnz), int(nfy), int(nfz), int(itime))
        _check(lib.senga_set_synthetic_inflow(self.h, C.byref(p)), "senga_set_synthetic_inflow")

    def set_transport(self, mixw=False, mixp=False, soret=False, dufour=False, wmltdr=5.0):
        """cont.dat transport switches: molar-mass and pressure diffusion,
        Soret and Dufour for species lighter than wmltdr (+1e-3)."""
        _check(lib.senga_set_transport(self.h, int(mixw), int(mixp), int(soret), int(dufour), float(wmltdr)),
               "senga_set_transport")

    def upload_async(self, fields, trun, itndex):
        """Queue the upload on the box's stream and return; the arrays (C
        contiguous, ideally page-locked) must stay alive and unchanged until
        sync()."""
        for a, dt in ((fields, np.float64), (trun, np.float64), (itndex, np.int32)):
            assert a.dtype == dt and a.flags.c_contiguous
        assert fields.shape == (self.nc,) + self.shape and trun.shape == self.shape
        assert itndex.shape == itn_shape(self.nspec, self.shape)
        _check(lib.senga_upload_state_async(self.h, _dp(fields), _dp(trun),
                                            itndex.ctypes.data_as(C.POINTER(C.c_int32))), "senga_upload_state_async")

    def download_async(self, fields, trun, itndex):
        """Queue the download into caller arrays and return; read them after
        sync()."""
        for a, dt in ((fields, np.float64), (trun, np.float64), (itndex, np.int32)):
            assert a.dtype == dt and a.flags.c_contiguous and a.flags.writeable
        assert fields.shape == (self.nc,) + self.shape and trun.shape == self.shape
        assert itndex.shape == itn_shape(self.nspec, self.shape)
        _check(lib.senga_download_state_async(self.h, _dp(fields), _dp(trun),
                                              itndex.ctypes.data_as(C.POINTER(C.c_int32))), "senga_download_state_async")

    def keep_rates(self, on=True):
        """Keep each substage's CHRATE rates (RRTE) for post_fields."""
        _check(lib.senga_keep_rates(self.h, 1 if on else 0), "senga_keep_rates")

    def post_fields(self):
        """Post-processing record fields (7 + 2 nspec, nz, ny, nx): rho, u, v,
        w, E, T, p, Y_k, RRTE_k (needs keep_rates before the step)."""
        out = np.empty((7 + 2 * self.nspec,) + self.shape)
        _check(lib.senga_post_fields_host(self.h, _dp(out)), "senga_post_fields_host")
        return out

    def set_radiation(self, radn):
        """Optically thin radiation loss (RADCAL) on with a Radn, off with None."""
        _check(lib.senga_set_radiation(self.h, C.byref(radn.t) if radn is not None else None),
               "senga_set_radiation")

    def tstep(self):
        """(TSTEP, last ERRMAX, INDERR) of the adaptive controller."""
        t, e, i = C.c_double(), C.c_double(), C.c_int()
        _check(lib.senga_get_tstep(self.h, C.byref(t), C.byref(e), C.byref(i)), "senga_get_tstep")
        return t.value, e.value, i.value

    def filter(self, mode=0):
        """FLTREM on the U register (mode bit 0: flip TWFACT's sign; bit 1:
        also filter the S register)."""
        _check(lib.senga_filter(self.h, mode), "senga_filter")

    def filter_field(self, f, mode=0):
        a = np.ascontiguousarray(f, dtype=np.float64)
        assert a.shape == self.shape
        out = np.empty_like(a)
        _check(lib.senga_filter_field_host(self.h, mode, _dp(a), _dp(out)), "senga_filter_field_host")
        return out

    def dfbydx(self, f): return self.deriv(0, f)
    def dfbydy(self, f): return self.deriv(1, f)
    def dfbydz(self, f): return self.deriv(2, f)
    def d2fdx2(self, f): return self.deriv(3, f)
    def d2fdy2(self, f): return self.deriv(4, f)
    def d2fdz2(self, f): return self.deriv(5, f)
    def d2fdxy(self, f): return self.deriv(6, f)
    def d2fdxz(self, f): return self.deriv(7, f)
    def d2fdyz(self, f): return self.deriv(8, f)


def make_config(shape, lengths, tstep, nend=(NPERI,) * 6, adaptive=False, device=0):
    cfg = ConfigT()
    cfg.nx, cfg.ny, cfg.nz = shape
    cfg.xgdlen, cfg.ygdlen, cfg.zgdlen = lengths
    for i, v in enumerate(nend):
        cfg.nend[i] = v
    cfg.tstep = tstep
    cfg.adaptive = 1 if adaptive else 0
    cfg.device = device
    return cfg


class Batch:
    """Ensemble of independent periodic boxes advanced together (one persistent
    launch per kernel family per substage, RK step as one CUDA graph)."""

    def __init__(self, boxes, chem, diff, device=0):
        """boxes: list of (shape_xyz, lengths, tstep)."""
        self.chem, self.diff = chem, diff
        self.nc = 5 + chem.nspec
        self.shapes = [(s[2], s[1], s[0]) for s, _, _ in boxes]
        arr = (ConfigT * len(boxes))(*[make_config(s, l, dt, device=device) for s, l, dt in boxes])
        h = C.c_void_p()
        _check(lib.senga_batch_create(len(boxes), arr, C.byref(chem.t), C.byref(diff.t), device, C.byref(h)),
               "senga_batch_create")
        self.h = h

    def close(self):
        if self.h:
            lib.senga_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, i, fields, trun, itndex):
        f = np.ascontiguousarray(fields, dtype=np.float64)
        t = np.ascontiguousarray(trun, dtype=np.float64)
        it = np.ascontiguousarray(itndex, dtype=np.int32)
        assert f.shape == (self.nc,) + self.shapes[i]
        _check(lib.senga_batch_upload_host(self.h, i, _dp(f), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32))),
               "senga_batch_upload_host")

    def download(self, i):
        f = np.empty((self.nc,) + self.shapes[i])
        t = np.empty(self.shapes[i])
        it = np.empty(self.shapes[i], dtype=np.int32)
        _check(lib.senga_batch_download_host(self.h, i, _dp(f), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32))),
               "senga_batch_download_host")
        return f, t, it

    def step(self, nsteps=1):
        _check(lib.senga_batch_step(self.h, nsteps), "senga_batch_step")

    def sync(self):
        _check(lib.senga_batch_sync(self.h), "senga_batch_sync")

    def autotune(self):
        a, b = C.c_int(), C.c_int()
        _check(lib.senga_batch_autotune(self.h, C.byref(a), C.byref(b)), "senga_batch_autotune")
        return dict(grid_stencil=a.value, grid_thermo=b.value, **self.form())

    def form(self):
        """The substage form in use: persistent (one launch per substage and
        table of 64 boxes) or four launches, and its grid."""
        p, g = C.c_int(), C.c_int()
        _check(lib.senga_batch_form(self.h, C.byref(p), C.byref(g)), "senga_batch_form")
        return {"persistent": bool(p.value), "grid": g.value}

    @property
    def stream(self):
        return lib.senga_batch_stream(self.h)

    def status(self):
        s = C.c_int()
        _check(lib.senga_batch_status(self.h, C.byref(s)), "senga_batch_status")
        return s.value


class Server:
    """Continuous-batching request loop (admission by HBM footprint)."""

    def __init__(self, arena_bytes, chem, diff, device=0):
        self.chem, self.diff = chem, diff
        self.nc = 5 + chem.nspec
        self.shapes = {}
        h = C.c_void_p()
        _check(lib.senga_server_create(arena_bytes, C.byref(chem.t), C.byref(diff.t), device, C.byref(h)),
               "senga_server_create")
        self.h = h

    def close(self):
        if self.h:
            lib.senga_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_max_points(self, max_points):
        """Cap on the grid points advanced per tick (0: arena only)."""
        _check(lib.senga_server_set_max_points(self.h, int(max_points)), "senga_server_set_max_points")

    def submit(self, shape, lengths, tstep, fields, trun, itndex, nsteps):
        cfg = make_config(shape, lengths, tstep)
        f = np.ascontiguousarray(fields, dtype=np.float64)
        t = np.ascontiguousarray(trun, dtype=np.float64)
        it = np.ascontiguousarray(itndex, dtype=np.int32)
        rid = C.c_int()
        _check(lib.senga_server_submit(self.h, C.byref(cfg), _dp(f), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32)),
                                       nsteps, C.byref(rid)), "senga_server_submit")
        self.shapes[rid.value] = (shape[2], shape[1], shape[0])
        return rid.value

    def tick(self):
        n = C.c_int()
        _check(lib.senga_server_tick(self.h, C.byref(n)), "senga_server_tick")
        return n.value

    def result(self, rid):
        shp = self.shapes[rid]
        f = np.empty((self.nc,) + shp)
        t = np.empty(shp)
        it = np.empty(shp, dtype=np.int32)
        tm = np.empty(3)
        _check(lib.senga_server_result(self.h, rid, _dp(f), _dp(t), it.ctypes.data_as(C.POINTER(C.c_int32)), _dp(tm)),
               "senga_server_result")
        return f, t, it, tm

    def stats(self):
        a, p = C.c_int(), C.c_int()
        g, fb = C.c_int64(), C.c_int64()
        _check(lib.senga_server_stats(self.h, C.byref(a), C.byref(p), C.byref(g), C.byref(fb)), "senga_server_stats")
        return {"active": a.value, "pending": p.value, "gpsu": g.value, "free_bytes": fb.value}
