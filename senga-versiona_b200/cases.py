"""Initial conditions and the named workloads (host side, numpy).

The reference builds its initial state in INDATA/TURBIN/FLAMIN on the CPU;
this module is this project's own generator of the same kind of state:
  * a solenoidal random-phase velocity field with a Passot-Pouquet spectrum
    E(k) ~ (k/k0)^4 exp(-2 (k/k0)^2) (the form of src/espect.f:63-65), scaled
    to the requested u' and integral length scale (l = sqrt(2 pi)/k0 for this
    spectrum), seeded;
  * Gaussian hot kernels on a uniform premixed mixture at uniform pressure;
  * the conversion to conserved variables of src/indata.f:1233-1375
    (rho = p/(R_mix T), E = sum h_k Y_k - R_mix T + |u|^2/2, interval index
    ITNDEX located as at src/indata.f:1268-1290).
Inputs of the benchmarks are synthetic: no dataset is involved.
"""
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data")
CHEM_1STEP = os.path.join(DATA, "chem_1step.dat")
CHEM_H2 = os.path.join(DATA, "chem_h2.dat")
DIFF_H2 = os.path.join(DATA, "diff_h2.dat")
RADN_H2 = os.path.join(DATA, "radn_h2.dat")  # Planck-mean absorption of H2O

NPERI = 2


def interval_index(chem, T):
    """ITNDEX: base-4 digits (2 bits) per species holding the thermo interval
    of T, 15 species per 32-bit word; shaped like T up to 15 species, else
    (words,) + T.shape, words slowest."""
    nw = (chem.nspec + 14) // 15
    itn = np.zeros((nw,) + T.shape, dtype=np.int32)
    ntint = chem.table("ntint")
    tinthi = chem.table("tinthi")
    for s in range(chem.nspec):
        it = np.zeros(T.shape, dtype=np.int32)
        for k in range(ntint[s] - 1):
            it = np.where((it == k) & (T > tinthi[s, k]), k + 1, it)
        itn[s // 15] += it << (2 * (s % 15))
    return itn[0] if nw == 1 else itn


def interval_of(itn, s, grid_ndim):
    """Interval (0-based) of species s from an ITNDEX array over a grid of
    grid_ndim dimensions."""
    word = itn if itn.ndim == grid_ndim else itn[s // 15]
    return (word >> (2 * (s % 15))) & 3


def species_enthalpy(chem, s, T, itn):
    """h_k(T) per unit mass from AMASCH (src/indata.f:1320-1333)."""
    ncpoly = chem.table("ncpoly")
    ncenth = chem.table("ncenth")
    amasch = chem.table("amasch")
    it = interval_of(itn, s, T.ndim)
    h = np.zeros(T.shape)
    for k in np.unique(it):
        m = it == k
        np_ = ncpoly[s, k]
        c = amasch[s, k]
        f = np.full(m.sum(), c[np_ - 1])
        for icp in range(np_ - 1, 0, -1):
            f = f * T[m] + c[icp - 1]
        h[m] = c[ncenth[s, k] - 1] + f * T[m]
    return h


def conserved(chem, p, T, u, v, w, Y):
    """Primitive -> conserved (src/indata.f:1233-1375). Y: (nspec, ...)."""
    rg = chem.table("rgspec")
    rmix = np.zeros(T.shape)
    for s in range(chem.nspec):
        rmix = rmix + rg[s] * Y[s]
    st1 = rmix * T
    rho = p / st1
    itn = interval_index(chem, T)
    E = np.zeros(T.shape)
    for s in range(chem.nspec):
        E = E + species_enthalpy(chem, s, T, itn) * Y[s]
    E = E - st1 + 0.5 * (u * u + v * v + w * w)
    fields = np.empty((5 + chem.nspec,) + T.shape)
    fields[0] = rho
    fields[1] = rho * u
    fields[2] = rho * v
    fields[3] = rho * w
    fields[4] = rho * E
    for s in range(chem.nspec):
        fields[5 + s] = rho * Y[s]
    return fields, itn


def temperature_from_state(chem, fields, tlo=200.0, thi=4000.0, iters=60):
    """T and ITNDEX of a conserved state by bisection on
    E(T) = sum_k Y_k h_k(T) - R_mix T + |u|^2 / 2 (the robust inversion
    TEMPIN performs at start-up, src/tempin.f), for restart dumps, which
    carry no temperature."""
    rho = fields[0]
    Y = fields[5:5 + chem.nspec] / rho
    ke = 0.5 * (fields[1] ** 2 + fields[2] ** 2 + fields[3] ** 2) / (rho * rho)
    e = fields[4] / rho - ke
    rg = chem.table("rgspec")
    rmix = sum(rg[s] * Y[s] for s in range(chem.nspec))

    def energy(T):
        itn = interval_index(chem, T)
        return sum(species_enthalpy(chem, s, T, itn) * Y[s] for s in range(chem.nspec)) - rmix * T

    lo = np.full(rho.shape, tlo)
    hi = np.full(rho.shape, thi)
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        up = energy(mid) < e
        lo = np.where(up, mid, lo)
        hi = np.where(up, hi, mid)
    T = 0.5 * (lo + hi)
    return T, interval_index(chem, T)


def passot_pouquet(shape, lengths, uprime, lint, seed):
    """Solenoidal random-phase velocity (u, v, w) with a Passot-Pouquet
    spectrum, rms per component = uprime, integral scale lint [m]."""
    nz, ny, nx = shape
    dx = [lengths[0] / (nx - 1), lengths[1] / (ny - 1), lengths[2] / (nz - 1)]
    rng = np.random.default_rng(seed)
    kx = 2 * np.pi * np.fft.fftfreq(nx, d=dx[0])
    ky = 2 * np.pi * np.fft.fftfreq(ny, d=dx[1])
    kz = 2 * np.pi * np.fft.fftfreq(nz, d=dx[2])
    KZ, KY, KX = np.meshgrid(kz, ky, kx, indexing="ij")
    k2 = KX * KX + KY * KY + KZ * KZ
    k = np.sqrt(k2)
    k0 = math.sqrt(2.0 * math.pi) / lint
    with np.errstate(divide="ignore", invalid="ignore"):
        spec = (k / k0) ** 4 * np.exp(-2.0 * (k / k0) ** 2)
        amp = np.where(k > 0, np.sqrt(spec / (4.0 * np.pi * np.maximum(k2, 1e-300))), 0.0)
    comps = []
    for _ in range(3):
        ph = rng.uniform(0.0, 2.0 * np.pi, size=k.shape)
        comps.append(amp * np.exp(1j * ph) * rng.standard_normal(k.shape))
    # projection onto the plane normal to k (solenoidal)
    with np.errstate(divide="ignore", invalid="ignore"):
        dot = (comps[0] * KX + comps[1] * KY + comps[2] * KZ) / np.where(k2 > 0, k2, 1.0)
    comps = [comps[0] - dot * KX, comps[1] - dot * KY, comps[2] - dot * KZ]
    vel = [np.real(np.fft.ifftn(c)) for c in comps]
    rms = math.sqrt(sum(float(np.mean(c * c)) for c in vel) / 3.0)
    scale = uprime / rms if rms > 0 else 0.0
    return [c * scale for c in vel]


def hot_kernels(shape, lengths, centres, radius, t0, tpeak):
    """Sum of Gaussian temperature bumps, minimum-image (periodic) distance."""
    nz, ny, nx = shape
    d = [lengths[0] / (nx - 1), lengths[1] / (ny - 1), lengths[2] / (nz - 1)]
    per = [nx * d[0], ny * d[1], nz * d[2]]
    z, y, x = np.meshgrid(np.arange(nz) * d[2], np.arange(ny) * d[1], np.arange(nx) * d[0], indexing="ij")
    bump = np.zeros(shape)
    for (cx, cy, cz) in centres:
        ddx = np.abs(x - cx)
        ddx = np.minimum(ddx, per[0] - ddx)
        ddy = np.abs(y - cy)
        ddy = np.minimum(ddy, per[1] - ddy)
        ddz = np.abs(z - cz)
        ddz = np.minimum(ddz, per[2] - ddz)
        bump = np.maximum(bump, np.exp(-(ddx * ddx + ddy * ddy + ddz * ddz) / (radius * radius)))
    return t0 + (tpeak - t0) * bump


def stable_dt(chem, fields, T, lengths, shape, cfl=0.5):
    """Fixed dt = cfl * min(Delta) / max(|u_i| + c) of the state."""
    nz, ny, nx = shape
    dmin = min(lengths[0] / (nx - 1), lengths[1] / (ny - 1), lengths[2] / (nz - 1))
    rho = fields[0]
    rg = chem.table("rgspec")
    rmix = sum(rg[s] * fields[5 + s] / rho for s in range(chem.nspec))
    # frozen cp from the first cp coefficient band is enough for a CFL bound
    amascp = chem.table("amascp")
    itn = interval_index(chem, T)
    cp = np.zeros(T.shape)
    ncpoly = chem.table("ncpoly")
    for s in range(chem.nspec):
        it = interval_of(itn, s, T.ndim)
        for k in np.unique(it):
            m = it == k
            c = amascp[s, k]
            f = np.full(m.sum(), c[ncpoly[s, k] - 1])
            for icp in range(ncpoly[s, k] - 1, 0, -1):
                f = f * T[m] + c[icp - 1]
            cp[m] += f * fields[5 + s][m] / rho[m]
    gam = cp / (cp - rmix)
    c = np.sqrt(gam * rmix * T)
    umax = max(float(np.max(np.abs(fields[i] / rho) + c)) for i in (1, 2, 3))
    return cfl * dmin / umax


def ignition_box(shape_xyz, seed, uprime, tpeak, chem_path=CHEM_1STEP):
    """One ignition-kernel box of the batched/served workloads: one-step
    chemistry, premixed reactant at 300 K and 101325 Pa, a centred Gaussian
    kernel of radius 1 mm and peak tpeak, Passot-Pouquet turbulence of rms
    uprime and integral scale 1 mm; grid spacing that of the 32^3 case."""
    from senga import Chem

    nx, ny, nz = shape_xyz
    dx = 2.0 * math.pi * 1.0e-3 / 31.0
    lengths = (dx * (nx - 1), dx * (ny - 1), dx * (nz - 1))
    chem = Chem(chem_path)
    shp = (nz, ny, nx)
    centre = (lengths[0] / 2, lengths[1] / 2, lengths[2] / 2)
    T = hot_kernels(shp, lengths, [centre], 1.0e-3, 300.0, tpeak)
    Y = np.zeros((2,) + shp)
    Y[0] = 1.0
    u, v, w = passot_pouquet(shp, lengths, uprime, 1.0e-3, seed)
    p = np.full(shp, 101325.0)
    fields, itn = conserved(chem, p, T, u, v, w, Y)
    dt = stable_dt(chem, fields, T, lengths, shp)
    return dict(name="ensemble", shape=tuple(shape_xyz), lengths=lengths, chem=chem_path, diff=None,
                fields=fields, T=T, itn=itn, dt=dt, nend=(NPERI,) * 6)


def make_case(name, n=None, seed=1234, scale_n=None, shape=None, chem_reader=None):
    """Named workloads. Returns dict with shape (nx,ny,nz), lengths, chem/diff
    paths, fields (nc,nz,ny,nx), T, itn and a CFL-0.5 dt.

    ignition32  : 32^3 periodic, side 2 pi mm, 1-step R->P, T0=300 K,
                  p=101325 Pa, one Gaussian kernel r=1 mm peak 1800 K,
                  u'=1 m/s, l=1 mm.
    h2_kernels  : 256^3 periodic, 10 mm, H2/air stoichiometric at 800 K,
                  101325 Pa, 8 seeded kernels r=0.5 mm peak 1600 K, u'=4 m/s,
                  l=1.5 mm (the integral scale of the 128^3 flame case).
    ensemble    : one box of the batched ensemble (sizes from {32,48,64,96},
                  seeded u' in U[0.5,3] m/s, peak T in U[1400,2000] K), 1-step.
    flame_inout : 128^3, 10 mm, H2/air mixture-averaged; NSCBC I3 inflow at
                  x-left (u = 1.25 m/s, v = w = 0, unburnt density and
                  composition) and O1 outflow at x-right (p_inf = 1e5 Pa,
                  sigma = 0.287, eta = 1e-3); y, z periodic. A planar lean
                  (Y_H2 = 0.0116) premixed flame: tanh progress profile of
                  thickness 0.5 mm at x = 3 mm from 300 K to 1350 K, burnt
                  composition of complete H2 -> H2O conversion; mean flow
                  1.25 m/s plus Passot-Pouquet turbulence u' = 2 m/s,
                  l = 1.5 mm. The result carries "bc" for the face setup.
    wall_box    : 32^3, 10 mm, H2/air mixture-averaged; W1 adiabatic no-slip
                  walls on both x faces, y and z periodic. Two seeded hot
                  kernels (r = 1 mm, 800 K -> 1600 K, the h2_pool
                  composition) near either wall, Passot-Pouquet turbulence
                  u' = 2 m/s, l = 1.5 mm, damped by sin^2(pi x / L) so that
                  the velocity vanishes on the walls; uniform 101325 Pa.
                  The result carries "bc" for the face setup.
    h2_pool     : 32^3 periodic, 10 mm, H2/air mixture-averaged with a
                  radical pool: the h2_kernels layout (4 seeded kernels
                  r = 1 mm, 800 K -> 1600 K) with the kernels' composition
                  moving from stoichiometric unburnt towards a partially
                  burnt mixture holding H, O, OH, HO2, H2O2, and a 5%
                  sinusoidal pressure modulation, so that the molar-mass,
                  pressure, Soret and Dufour terms are all active.
    `n` overrides the grid extent (cubic) for smaller test instances;
    `shape` = (nx, ny, nz) gives h2_pool and flame_inout a non-cubic grid.
    `chem_reader` is the class that reads chem.dat (path -> object with
    nspec and table(name)); the default is the device library's Chem.
    """
    if chem_reader is None:
        from senga import Chem as chem_reader  # noqa: local import keeps this module numpy-only
    Chem = chem_reader
    rng = np.random.default_rng(seed)
    if name == "ignition32":
        nn = n or 32
        shape_xyz = (nn, nn, nn)
        L = 2.0 * math.pi * 1.0e-3
        lengths = (L, L, L)
        chem_path, diff_path = CHEM_1STEP, None
        chem = Chem(chem_path)
        shp = (nn, nn, nn)
        T = hot_kernels(shp, lengths, [(L / 2, L / 2, L / 2)], 1.0e-3, 300.0, 1800.0)
        Y = np.zeros((2,) + shp)
        Y[0] = 1.0
        u, v, w = passot_pouquet(shp, lengths, 1.0, 1.0e-3, seed)
        p = np.full(shp, 101325.0)
    elif name == "h2_kernels":
        nn = n or 256
        shape_xyz = (nn, nn, nn)
        L = 1.0e-2
        lengths = (L, L, L)
        chem_path, diff_path = CHEM_H2, DIFF_H2
        chem = Chem(chem_path)
        shp = (nn, nn, nn)
        centres = [tuple(rng.uniform(0.0, L, size=3)) for _ in range(8)]
        T = hot_kernels(shp, lengths, centres, 0.5e-3, 800.0, 1600.0)
        wm = chem.table("wmolar")
        # stoichiometric H2/air: 2 H2 + O2 + 3.76 N2 (species 1 H2, 2 O2, 9 N2)
        mass = np.array([2 * wm[0], wm[1], 3.76 * wm[8]])
        yv = mass / mass.sum()
        Y = np.zeros((9,) + shp)
        Y[0], Y[1], Y[8] = yv[0], yv[1], yv[2]
        u, v, w = passot_pouquet(shp, lengths, 4.0, 1.5e-3, seed)
        p = np.full(shp, 101325.0)
    elif name == "flame_inout":
        nn = n or 128
        shape_xyz = tuple(shape) if shape else (nn, nn, nn)
        L = 1.0e-2
        lengths = (L, L, L)
        chem_path, diff_path = CHEM_H2, DIFF_H2
        chem = Chem(chem_path)
        shp = shape_xyz[::-1]
        wm = chem.table("wmolar")
        yu = np.zeros(9)
        yu[0], yu[1], yu[8] = 1.1606960e-2, 2.30295282e-1, 7.58097758e-1  # input/cont.dat defaults
        yb = yu.copy()
        nh2 = yu[0] / wm[0]
        yb[0] = 0.0
        yb[1] = yu[1] - 0.5 * nh2 * wm[1]
        yb[2] = nh2 * wm[2]
        x = np.arange(shape_xyz[0]) * (L / (shape_xyz[0] - 1))
        prog = 0.5 * (1.0 + np.tanh((x - 3.0e-3) / 0.5e-3))
        prog3 = np.broadcast_to(prog, shp)
        T = 300.0 + (1350.0 - 300.0) * prog3
        Y = np.array([yu[k] + (yb[k] - yu[k]) * prog3 for k in range(9)])
        u, v, w = passot_pouquet(shp, lengths, 2.0, 1.5e-3, seed)
        u = u + 1.25
        p = np.full(shp, 1.0e5)
        fields, itn = conserved(chem, p, T, u, v, w, Y)
        rg = chem.table("rgspec")
        rho_in = 1.0e5 / (300.0 * float(sum(rg[k] * yu[k] for k in range(9))))
        bc = dict(xl=13, xr=21, u_in=1.25, rho_in=rho_in, y_in=tuple(float(v_) for v_ in yu), p_inf=1.0e5,
                  sigma=0.287, eta=1.0e-3, pio=0, bet_local=0)
        dt = stable_dt(chem, fields, T, lengths, shp)
        return dict(name=name, shape=shape_xyz, lengths=lengths, chem=chem_path, diff=diff_path, fields=fields, T=T,
                    itn=itn, dt=dt, nend=(1, 1, NPERI, NPERI, NPERI, NPERI), bc=bc)
    elif name == "wall_box":
        nn = n or 32
        shape_xyz = tuple(shape) if shape else (nn, nn, nn)
        L = 1.0e-2
        lengths = (L, L, L)
        chem_path, diff_path = CHEM_H2, DIFF_H2
        chem = Chem(chem_path)
        shp = shape_xyz[::-1]
        centres = [(rng.uniform(0.5e-3, 2.0e-3), rng.uniform(0.0, L), rng.uniform(0.0, L)),
                   (L - rng.uniform(1.0e-3, 3.0e-3), rng.uniform(0.0, L), rng.uniform(0.0, L))]
        T = hot_kernels(shp, lengths, centres, 1.0e-3, 800.0, 1600.0)
        prog = (T - 800.0) / 800.0
        wm = chem.table("wmolar")
        mass = np.array([2 * wm[0], wm[1], 3.76 * wm[8]])
        yu = np.zeros(9)
        yu[0], yu[1], yu[8] = mass / mass.sum()
        yb = np.array([0.01, 0.12, 0.14, 0.004, 0.012, 0.002, 0.0005, 0.0002, 0.0])
        yb[8] = 1.0 - yb[:8].sum()
        Y = np.array([yu[k] + (yb[k] - yu[k]) * prog for k in range(9)])
        u, v, w = passot_pouquet(shp, lengths, 2.0, 1.5e-3, seed)
        x = np.arange(shape_xyz[0]) * (L / (shape_xyz[0] - 1))
        damp = np.broadcast_to(np.sin(math.pi * x / L) ** 2, shp)
        damp = np.where(np.abs(damp) < 1e-30, 0.0, damp)
        u, v, w = u * damp, v * damp, w * damp
        for a in (u, v, w):
            a[..., 0] = 0.0
            a[..., -1] = 0.0
        p = np.full(shp, 101325.0)
        fields, itn = conserved(chem, p, T, u, v, w, Y)
        dt = stable_dt(chem, fields, T, lengths, shp)
        return dict(name=name, shape=shape_xyz, lengths=lengths, chem=chem_path, diff=diff_path, fields=fields, T=T,
                    itn=itn, dt=dt, nend=(1, 1, NPERI, NPERI, NPERI, NPERI), bc=dict(xl=31, xr=31))
    elif name == "h2_pool":
        nn = n or 32
        shape_xyz = tuple(shape) if shape else (nn, nn, nn)
        L = 1.0e-2
        lengths = (L, L, L)
        chem_path, diff_path = CHEM_H2, DIFF_H2
        chem = Chem(chem_path)
        shp = shape_xyz[::-1]
        centres = [tuple(rng.uniform(0.0, L, size=3)) for _ in range(4)]
        T = hot_kernels(shp, lengths, centres, 1.0e-3, 800.0, 1600.0)
        prog = (T - 800.0) / 800.0
        wm = chem.table("wmolar")
        mass = np.array([2 * wm[0], wm[1], 3.76 * wm[8]])
        yu = np.zeros(9)
        yu[0], yu[1], yu[8] = mass / mass.sum()
        yb = np.array([0.01, 0.12, 0.14, 0.004, 0.012, 0.002, 0.0005, 0.0002, 0.0])
        yb[8] = 1.0 - yb[:8].sum()
        Y = np.array([yu[k] + (yb[k] - yu[k]) * prog for k in range(9)])
        u, v, w = passot_pouquet(shp, lengths, 2.0, 1.5e-3, seed)
        z_, y_, x_ = np.meshgrid(*(np.arange(m) * (L / (m - 1)) for m in shp), indexing="ij")
        p = 101325.0 * (1.0 + 0.05 * np.sin(2 * math.pi * x_ / L) * np.sin(2 * math.pi * y_ / L))
    elif name == "ensemble":
        sizes = (32, 48, 64, 96)
        shape_xyz = tuple(int(rng.choice(sizes)) for _ in range(3)) if n is None else (n, n, n)
        up = float(rng.uniform(0.5, 3.0))
        tpk = float(rng.uniform(1400.0, 2000.0))
        return ignition_box(shape_xyz, seed, up, tpk)
    else:
        raise ValueError(f"unknown case {name}")
    fields, itn = conserved(chem, p, T, u, v, w, Y)
    nx, ny, nz = shape_xyz
    dt = stable_dt(chem, fields, T, lengths, (nz, ny, nx))
    return dict(name=name, shape=shape_xyz, lengths=lengths, chem=chem_path, diff=diff_path,
                fields=fields, T=T, itn=itn, dt=dt, nend=(NPERI,) * 6)
