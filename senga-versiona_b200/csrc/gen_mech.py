"""Generates mech_gen.cuh: straight-line per-point thermochemistry for the
mechanisms shipped in ../data (the 21-step H2/air mechanism with its
mixture-averaged transport data, and the single-step R -> P mechanism with
constant-Lewis transport).

Each mechanism becomes a policy struct (same interface as MechTables in
kernels.cu) in which every table value is a hex-float literal and every loop
over species, reaction steps and polynomial coefficients is unrolled. The
derived tables are computed here with the same IEEE operations, in the same
order, as the host loader (tables_host.cpp, restating src/chemin.f:822-983
and src/diffin.f:328-405); a generated host function `matches()` compares
every literal against the tables actually loaded at run time, and the
generated policy is used only when all are bit-identical.

Usage: python gen_mech.py <out.cuh>
"""
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(os.path.dirname(HERE), "data")
RGUNIV = 8.3142e3
ALAMDC, RLAMDA, TLAMDA = 2.58e-5, 7.0e-1, 2.98e2
DFCTOL = 1.0e-12


def h(x):
    """C++ hex-float literal of a Python float (exact)."""
    x = float(x)
    if x == 0.0:
        return "0.0"
    return x.hex().replace("0x", "0x") if x > 0 else "-" + (-x).hex()


def fld(rec, col, width):
    return "".join(ch for ch in rec[col:col + width] if ch not in " \t").replace("D", "E").replace("d", "E")


def ifld(rec, col, width):
    s = fld(rec, col, width)
    return int(s) if s else 0


def rfld(rec, col, width):
    s = fld(rec, col, width)
    return float(s) if s else 0.0


def free(rec):
    return [float(t.replace("D", "E").replace("d", "E")) for t in rec.replace(",", " ").split()]


class Lines:
    def __init__(self, path):
        with open(path) as fh:
            self.l = [x.rstrip("\r\n") for x in fh]
        self.i = 0

    def next(self):
        self.i += 1
        return self.l[self.i - 1]

    def skip(self, n=1):
        self.i += n


def load_chem(path):
    r = Lines(path)
    r.skip(6)
    ns = ifld(r.next(), 0, 5)
    r.skip(ns + 1)
    c = dict(nspec=ns, prefgb=free(r.next())[0], wmolar=[0.0] * ns, clewis=[0.0] * ns, ntint=[0] * ns,
             tinthi=[[0.0, 0.0] for _ in range(ns)], ncofcp=[[0, 0] for _ in range(ns)],
             amolcp=[[[0.0] * 7 for _ in range(2)] for _ in range(ns)])
    for _ in range(ns):
        rec = r.next()
        s = ifld(rec, 0, 5) - 1
        c["wmolar"][s] = rfld(rec, 5, 12)
        c["clewis"][s] = rfld(r.next(), 0, 12)
        c["ntint"][s] = ifld(r.next(), 0, 5)
        for it in range(c["ntint"][s]):
            ri = r.next()
            c["tinthi"][s][it] = rfld(ri, 12, 12)
            c["ncofcp"][s][it] = ifld(ri, 24, 5)
            for q in range(c["ncofcp"][s][it]):
                c["amolcp"][s][it][q] = rfld(r.next(), 0, 15)
    r.skip()
    nst = ifld(r.next(), 0, 5)
    c["nstep"] = nst
    c["rparam"] = [[0.0] * 3 for _ in range(nst)]
    for _ in range(nst):
        rec = r.next()
        st = ifld(rec, 0, 5) - 1
        c["rparam"][st] = [rfld(rec, 5 + 12 * q, 12) for q in range(3)]

    def step_list(with_coef):
        r.skip()
        lst = [[] for _ in range(nst)]
        for _ in range(nst):
            rec = r.next()
            st = ifld(rec, 0, 5) - 1
            ln = ifld(rec, 5, 5)
            entries = []
            for _ in range(ln):
                e = r.next()
                entries.append((ifld(e, 5, 5) - 1, ifld(e, 10, 8), rfld(e, 18, 12) if with_coef else None))
            entries.sort()
            lst[st] = [(sp, cf) for _, sp, cf in entries]
        return lst

    c["nsspec"] = step_list(False)
    c["nrspec"] = step_list(False)
    c["npspec"] = step_list(False)
    c["nrcpec"] = step_list(True)
    c["npcpec"] = step_list(True)
    r.skip()
    c["diffmu"] = [[0.0] * len(c["nsspec"][st]) for st in range(nst)]
    for st in range(nst):
        for _ in range(len(c["nsspec"][st])):
            e = r.next()
            c["diffmu"][ifld(e, 0, 5) - 1][ifld(e, 5, 5) - 1] = rfld(e, 10, 5)
    r.skip()
    nb = ifld(r.next(), 0, 5)
    c["nbody"] = nb
    r.skip(nb + 1)
    c["mblist"] = [0] * nst
    if nb > 0:
        for _ in range(nst):
            e = r.next()
            c["mblist"][ifld(e, 0, 5) - 1] = ifld(e, 5, 8)
    r.skip()
    c["effy3b"] = [[0.0] * ns for _ in range(max(nb, 1))]
    for _ in range(nb * ns):
        e = r.next()
        c["effy3b"][ifld(e, 0, 5) - 1][ifld(e, 5, 5) - 1] = rfld(e, 10, 12)

    def flag_list():
        r.skip()
        cnt = ifld(r.next(), 0, 5)
        lst = [0] * nst
        if cnt > 0:
            for _ in range(nst):
                e = r.next()
                lst[ifld(e, 0, 5) - 1] = ifld(e, 5, 8)
        return cnt, lst

    c["ngibb"], c["mglist"] = flag_list()
    c["nlind"], c["mllist"] = flag_list()
    r.skip()
    c["rclind"] = []
    for _ in range(c["nlind"]):
        e = r.next()
        c["rclind"].append([rfld(e, 5 + 12 * q, 12) for q in range(4)])
    c["ntroe"], c["mtlist"] = flag_list()
    r.skip()
    if c["ntroe"]:
        raise NotImplementedError("Troe steps: use the table-driven path")
    c["nsrif"], c["mslist"] = flag_list()
    if c["nsrif"]:
        raise NotImplementedError("SRI steps: use the table-driven path")
    # ---- derived (src/chemin.f:822-983; same operations as tables_host.cpp) ----
    for st in range(nst):
        c["rparam"][st][0] = math.log(c["rparam"][st][0])
        c["rparam"][st][2] = c["rparam"][st][2] / RGUNIV
    for L in c["rclind"]:
        L[0] = math.log(L[0])
        L[2] = L[2] / RGUNIV
    c["diffmw"] = [[c["diffmu"][st][q] * c["wmolar"][c["nsspec"][st][q][0] - 1] for q in range(len(c["nsspec"][st]))]
                   for st in range(nst)]
    c["ovwmol"] = [1.0 / w for w in c["wmolar"]]
    c["rgspec"] = [RGUNIV * o for o in c["ovwmol"]]
    c["amascp"] = [[[0.0] * 7 for _ in range(2)] for _ in range(ns)]
    c["amasct"] = [[[0.0] * 7 for _ in range(2)] for _ in range(ns)]
    c["amasch"] = [[[0.0] * 7 for _ in range(2)] for _ in range(ns)]
    c["amolgb"] = [[[0.0] * 7 for _ in range(2)] for _ in range(ns)]
    c["ncpoly"] = [[0, 0] for _ in range(ns)]
    c["ncenth"] = [[0, 0] for _ in range(ns)]
    c["ncenpy"] = [[0, 0] for _ in range(ns)]
    for s in range(ns):
        for it in range(c["ntint"][s]):
            ncof = c["ncofcp"][s][it]
            np_, nh, nsy = ncof - 2, ncof - 1, ncof
            c["ncpoly"][s][it], c["ncenth"][s][it], c["ncenpy"][s][it] = np_, nh, nsy
            cp = [c["amolcp"][s][it][q] * RGUNIV * c["ovwmol"][s] for q in range(ncof)] + [0.0] * (7 - ncof)
            c["amascp"][s][it] = cp
            t = [0.0] * 7
            hh = [0.0] * 7
            t[0] = cp[0] - c["rgspec"][s]
            hh[0] = cp[0]
            for q in range(2, np_ + 1):
                t[q - 1] = cp[q - 1] / float(q)
                hh[q - 1] = cp[q - 1] / float(q)
            t[nh - 1] = 0.0
            t[nsy - 1] = 0.0
            hh[nh - 1] = cp[nh - 1]
            hh[nsy - 1] = 0.0
            c["amasct"][s][it] = t
            c["amasch"][s][it] = hh
    giblet = math.log(c["prefgb"] / RGUNIV)
    for s in range(ns):
        for it in range(c["ntint"][s]):
            m = c["amolcp"][s][it]
            np_, nh, nsy = c["ncpoly"][s][it], c["ncenth"][s][it], c["ncenpy"][s][it]
            g = [0.0] * 7
            g[0] = m[nsy - 1] - m[0] + giblet
            for q in range(2, np_ + 1):
                g[q - 1] = m[q - 1] / float(q * (q - 1))
            g[nh - 1] = m[nh - 1]
            g[nsy - 1] = m[0] - 1.0
            c["amolgb"][s][it] = g
    c["olewis"] = [1.0 / x for x in c["clewis"]]
    c["alamda"] = ALAMDC * math.exp(-RLAMDA * math.log(TLAMDA))
    return c


def load_diff(path, c):
    r = Lines(path)
    r.skip(6)
    ns = ifld(r.next(), 0, 5)
    r.skip(ns + 1)
    v = free(r.next())
    d = dict(pdifgb=v[0], tdifgb=v[1])

    def values(n):
        out = []
        while len(out) < n:
            out += free(r.next())
        return out

    r.skip()
    d["viscco"] = []
    for _ in range(ns):
        d["ncovis"] = int(free(r.next())[1])
        d["viscco"].append(values(d["ncovis"]))
    r.skip()
    d["condco"] = []
    for _ in range(ns):
        d["ncocon"] = int(free(r.next())[1])
        d["condco"].append(values(d["ncocon"]))
    r.skip()
    d["diffco"] = [[None] * ns for _ in range(ns)]
    for s in range(ns):
        d["ncodif"] = int(free(r.next())[1])
        for t in range(s + 1):
            d["diffco"][s][t] = values(1 + d["ncodif"])[1:]
    for s in range(ns):
        for t in range(s + 1, ns):
            d["diffco"][s][t] = d["diffco"][t][s]
    w = c["wmolar"]
    d["wilko2"] = [[1.0 / math.sqrt(math.sqrt(w[s] / w[t])) for t in range(ns)] for s in range(ns)]
    d["wilko1"] = [[1.0 / math.sqrt(8.0 * (1.0 + w[s] / w[t])) for t in range(ns)] for s in range(ns)]
    return d


def poly_expr(coefs, var):
    """Horner in the reference order: f = c[n-1]; f = f*var + c[k]."""
    e = h(coefs[-1])
    for k in range(len(coefs) - 2, -1, -1):
        e = f"({e} * {var} + {h(coefs[k])})"
    return e


def sel(it_var, a, b):
    return a if a == b else f"({it_var} ? {b} : {a})"


def gen(tag, c, d):
    ns = c["nspec"]
    mavt = d is not None
    o = []
    w = o.append
    w(f"struct Mech_{tag} {{")
    w(f"  static constexpr int NS = {ns};")
    w(f"  static constexpr bool MAVT = {'true' if mavt else 'false'};")
    w("  __device__ __forceinline__ bool has(int) const { return true; }")
    w("  __device__ __forceinline__ int count() const { return NS; }")
    # ---- temper coefficients
    w("  __device__ __forceinline__ void temper_coeffs(const double (&ry)[NS], uint64_t itn0, double (&tc)[6], double (&td)[6], double& rmix) const {")
    for s in range(ns):
        w(f"    {{ const int it = (itn0 >> {2 * s}) & 1; const double y = ry[{s}];")
        nint = c["ntint"][s]
        def cv(table, q):
            a = table[s][0][q]
            b = table[s][1][q] if nint > 1 else a
            return sel("it", h(a), h(b))
        nh = c["ncenth"][s][0]
        np_ = c["ncpoly"][s][0]
        if nint > 1 and (c["ncenth"][s][1] != nh or c["ncpoly"][s][1] != np_):
            raise NotImplementedError("interval-dependent polynomial length")
        w(f"      tc[0] = tc[0] + y * {cv(c['amascp'], nh - 1)};")
        w(f"      tc[1] = tc[1] + y * {cv(c['amasct'], 0)};")
        w("      td[1] = tc[1];")
        for icp in range(2, np_ + 1):
            w(f"      tc[{icp}] = tc[{icp}] + y * {cv(c['amasct'], icp - 1)};")
            w(f"      td[{icp}] = td[{icp}] + y * {cv(c['amascp'], icp - 1)};")
        w(f"      rmix = rmix + y * {h(c['rgspec'][s])}; }}")
    w("  }")
    # ---- locate + cp
    w("  __device__ __forceinline__ void locate(double T, const double (&ry)[NS], uint64_t& itn, double& cpsum) const {")
    w("    itn = 0; cpsum = 0.0;")
    for s in range(ns):
        np_ = c["ncpoly"][s][0]
        if c["ntint"][s] > 1:
            w(f"    {{ const int it = T > {h(c['tinthi'][s][0])} ? 1 : 0; itn += (uint64_t)it << {2 * s};")
        else:
            w("    { const int it = 0; (void)it;")
        cp0, cp1 = c["amascp"][s][0], (c["amascp"][s][1] if c["ntint"][s] > 1 else c["amascp"][s][0])
        w(f"      double v = {sel('it', h(cp0[np_ - 1]), h(cp1[np_ - 1]))};")
        for icp in range(np_ - 1, 0, -1):
            w(f"      v = v * T + {sel('it', h(cp0[icp - 1]), h(cp1[icp - 1]))};")
        w(f"      cpsum = cpsum + ry[{s}] * v; }}")
    w("  }")
    w(f"  __device__ __forceinline__ double alamda() const {{ return {h(c['alamda'])}; }}")
    w("  __device__ __forceinline__ double olewis(int s) const {")
    w("    switch (s) {")
    for s in range(ns):
        w(f"      case {s}: return {h(c['olewis'][s])};")
    w("      default: return 0.0; }")
    w("  }")
    # ---- mixture-averaged transport
    w("  __device__ __forceinline__ void mixture(double T, double p, double rho, const double (&ry)[NS], const double (&y)[NS], double& lam, double (&rd)[NS], double& mu) const {")
    if mavt:
        w(f"    const double lt = log(T / {h(d['tdifgb'])});")
        w("    double c1 = 0.0, c2 = 0.0, c3 = 0.0;")
        for s in range(ns):
            w(f"    {{ const double lk = exp({poly_expr(d['condco'][s], 'lt')}); const double fm = ry[{s}] * {h(c['ovwmol'][s])};")
            w("      c1 = c1 + fm * lk; c2 = c2 + fm / lk; c3 = c3 + fm; }")
        w("    c3 = 1.0 / c3; c1 = c1 * c3; c2 = c2 * c3;")
        w("    lam = 0.5 * (c1 + 1.0 / c2);")
        w("    const double wmix = rho * c3;")
        w(f"    const double povr = p / {h(d['pdifgb'])};")
        # Wilke viscosity before the mixture diffusivities, so that the nine
        # rho D_k are formed last and stored right after: the square roots
        # and the diffusivity sums are never live together (fewer registers);
        # mu_k is taken as sqrt(mu_k)^2 (within an ulp of mu_k)
        for s in range(ns):
            w(f"    const double sq{s} = sqrt(exp({poly_expr(d['viscco'][s], 'lt')})); const double rq{s} = 1.0 / sq{s};")
        w("    mu = 0.0;")
        for s in range(ns):
            w("    { double cc = 0.0, fw;")
            for t in range(ns):
                w(f"      fw = 1.0 + sq{s} * rq{t} * {h(d['wilko2'][s][t])}; fw = {h(d['wilko1'][s][t])} * fw * fw; cc = cc + y[{t}] * {h(c['ovwmol'][t])} * fw;")
            w(f"      mu = mu + y[{s}] * {h(c['ovwmol'][s])} * ((sq{s} * sq{s}) / cc); }}")
        w("    double sumy = 0.0;")
        for s in range(ns):
            w(f"    sumy += y[{s}] + {h(DFCTOL)};")
        for s in range(ns):
            w(f"    double den{s} = 0.0;")
        for s in range(ns):
            for t in range(s + 1, ns):
                w(f"    {{ const double inv = exp(-{poly_expr(d['diffco'][s][t], 'lt')}) * povr;")
                w(f"      den{s} += (y[{t}] + {h(DFCTOL)}) * {h(c['ovwmol'][t])} * inv;")
                w(f"      den{t} += (y[{s}] + {h(DFCTOL)}) * {h(c['ovwmol'][s])} * inv; }}")
        for s in range(ns):
            w(f"    rd[{s}] = rho * (sumy - (y[{s}] + {h(DFCTOL)})) / (den{s} * wmix);")
    else:
        w("    (void)T; (void)p; (void)rho; (void)ry; (void)y; lam = 0.0; mu = 0.0;")
        w("    for (int s = 0; s < NS; ++s) rd[s] = 0.0;")
    w("  }")
    # ---- enthalpy
    w("  __device__ __forceinline__ void enthalpy(double T, uint64_t itn, double (&hk)[NS]) const {")
    for s in range(ns):
        np_, nh = c["ncpoly"][s][0], c["ncenth"][s][0]
        a0 = c["amasch"][s][0]
        a1 = c["amasch"][s][1] if c["ntint"][s] > 1 else a0
        w(f"    {{ const int it = (itn >> {2 * s}) & 1; (void)it; double v = {sel('it', h(a0[np_ - 1]), h(a1[np_ - 1]))};")
        for icp in range(np_ - 1, 0, -1):
            w(f"      v = v * T + {sel('it', h(a0[icp - 1]), h(a1[icp - 1]))};")
        w(f"      hk[{s}] = {sel('it', h(a0[nh - 1]), h(a1[nh - 1]))} + v * T; }}")
    w("  }")
    # ---- CHRATE
    w("  __device__ __forceinline__ void chrate(double T, uint64_t itn, const double (&ry)[NS], double (&rate)[NS]) const {")
    w("    const double lnT = log(T); const double ovT = 1.0 / T; (void)itn;")
    for s in range(ns):
        w(f"    rate[{s}] = 0.0;")
    need_gibbs = c["ngibb"] > 0
    if need_gibbs:
        for s in range(ns):
            np_, nh, nsy = c["ncpoly"][s][0], c["ncenth"][s][0], c["ncenpy"][s][0]
            g0 = c["amolgb"][s][0]
            g1 = c["amolgb"][s][1] if c["ntint"][s] > 1 else g0
            w(f"    double gib{s}; {{ const int it = (itn >> {2 * s}) & 1; (void)it; double v = {sel('it', h(g0[np_ - 1]), h(g1[np_ - 1]))};")
            for icp in range(np_ - 1, 0, -1):
                w(f"      v = {sel('it', h(g0[icp - 1]), h(g1[icp - 1]))} + v * T;")
            w(f"      gib{s} = {sel('it', h(g0[nh - 1]), h(g1[nh - 1]))} / T - {sel('it', h(g0[nsy - 1]), h(g1[nsy - 1]))} * lnT - v; }}")
    w("    double s3 = 0.0; (void)s3;")
    for st in range(c["nstep"]):
        w(f"    {{ // step {st + 1}")
        ib = c["mblist"][st]
        flthrd = True
        if ib != 0:
            terms = " + ".join(f"ry[{s}] * {h(c['ovwmol'][s] * c['effy3b'][ib - 1][s])}" for s in range(ns))
            w("      s3 = 0.0;")
            for s in range(ns):
                w(f"      s3 += ry[{s}] * {h(c['ovwmol'][s] * c['effy3b'][ib - 1][s])};")
        A, nexp, E = c["rparam"][st]
        w(f"      double s2 = {h(A)} + {h(nexp)} * lnT - {h(E)} * ovT;")
        w("      double s1 = exp(s2);")
        if c["mllist"][st] != 0:
            L = c["rclind"][c["mllist"][st] - 1]
            import struct
            flc = struct.unpack("f", struct.pack("f", L[3]))[0]  # REAL (single) in the reference
            w(f"      {{ const double s4 = exp({h(L[0])} + {h(L[1])} * lnT - {h(L[2])} * ovT);")
            w("        const double pr = s3 * s4 / s1;")
            w(f"        s1 = s1 * ({h(flc)} * pr / (1.0 + pr)); s2 = log(s1); }}")
            flthrd = False
        for sp, _ in c["nrspec"][st]:
            w(f"      s1 = s1 * fmax(ry[{sp - 1}] * {h(c['ovwmol'][sp - 1])}, 0.0);")
        for sp, cf in c["nrcpec"][st]:
            w(f"      {{ double fn = fmax(ry[{sp - 1}] * {h(c['ovwmol'][sp - 1])}, 1.0e-30); fn = exp({h(cf)} * log(fn)); s1 = s1 * (fn / (1.0 + 1.0e-15 * fn)); }}")
        if c["mglist"][st] != 0:
            for q, (sp, _) in enumerate(c["nsspec"][st]):
                w(f"      s2 = s2 + {h(c['diffmu'][st][q])} * gib{sp - 1};")
            w("      s2 = exp(s2);")
            for sp, _ in c["npspec"][st]:
                w(f"      s2 = s2 * fmax(ry[{sp - 1}] * {h(c['ovwmol'][sp - 1])}, 0.0);")
            for sp, cf in c["npcpec"][st]:
                w(f"      {{ double fn = fmax(ry[{sp - 1}] * {h(c['ovwmol'][sp - 1])}, 1.0e-30); fn = exp({h(cf)} * log(fn)); s2 = s2 * (fn / (1.0 + 1.0e-15 * fn)); }}")
            w("      s1 = s1 - s2;")
        else:
            w("      (void)s2;")
        if ib != 0 and flthrd:
            w("      s1 = s1 * s3;")
        for q, (sp, _) in enumerate(c["nsspec"][st]):
            w(f"      rate[{sp - 1}] += s1 * {h(c['diffmw'][st][q])};")
        w("    }")
    w("  }")
    # ---- host-side exact match against the loaded tables
    w("  static bool matches(const senga_chem& C, const senga_diff& D) {")
    w("    bool ok = true;")
    w(f"    ok = ok && C.nspec == {ns} && C.nstep == {c['nstep']} && C.ntroe == 0 && C.nsrif == 0;")
    w(f"    ok = ok && C.nbody == {c['nbody']} && C.nlind == {c['nlind']} && C.ngibb == {c['ngibb']};")
    w(f"    ok = ok && D.flmavt == {1 if mavt else 0};")
    w(f"    ok = ok && C.alamda == {h(c['alamda'])};")
    for s in range(ns):
        w(f"    ok = ok && C.ntint[{s}] == {c['ntint'][s]} && C.rgspec[{s}] == {h(c['rgspec'][s])} && C.ovwmol[{s}] == {h(c['ovwmol'][s])} && C.olewis[{s}] == {h(c['olewis'][s])};")
        for it in range(c["ntint"][s]):
            w(f"    ok = ok && C.ncpoly[{s}][{it}] == {c['ncpoly'][s][it]} && C.ncenth[{s}][{it}] == {c['ncenth'][s][it]} && C.ncenpy[{s}][{it}] == {c['ncenpy'][s][it]};")
            if it == 0 and c["ntint"][s] > 1:
                w(f"    ok = ok && C.tinthi[{s}][0] == {h(c['tinthi'][s][0])};")
            for q in range(7):
                for tb in ("amascp", "amasct", "amasch", "amolgb"):
                    w(f"    ok = ok && C.{tb}[{s}][{it}][{q}] == {h(c[tb][s][it][q])};")
    for st in range(c["nstep"]):
        for q in range(3):
            w(f"    ok = ok && C.rparam[{st}][{q}] == {h(c['rparam'][st][q])};")
        w(f"    ok = ok && C.mblist[{st}] == {c['mblist'][st]} && C.mglist[{st}] == {c['mglist'][st]} && C.mllist[{st}] == {c['mllist'][st]} && C.mtlist[{st}] == 0 && C.mslist[{st}] == 0;")
        for nm, key in (("nsslen", "nsspec"), ("nrslen", "nrspec"), ("npslen", "npspec"), ("nrclen", "nrcpec"), ("npclen", "npcpec")):
            w(f"    ok = ok && C.{nm}[{st}] == {len(c[key][st])};")
            for q, (sp, cf) in enumerate(c[key][st]):
                w(f"    ok = ok && C.{key}[{st}][{q}] == {sp};")
                if cf is not None:
                    w(f"    ok = ok && C.{'crspec' if key == 'nrcpec' else 'cpspec'}[{st}][{q}] == {h(cf)};")
        for q in range(len(c["nsspec"][st])):
            w(f"    ok = ok && C.diffmu[{st}][{q}] == {h(c['diffmu'][st][q])} && C.diffmw[{st}][{q}] == {h(c['diffmw'][st][q])};")
    for b in range(c["nbody"]):
        for s in range(ns):
            w(f"    ok = ok && C.effy3b[{b}][{s}] == {h(c['effy3b'][b][s])};")
    for i, L in enumerate(c["rclind"]):
        for q in range(4):
            w(f"    ok = ok && C.rclind[{i}][{q}] == {h(L[q])};")
    if mavt:
        w(f"    ok = ok && D.tdifgb == {h(d['tdifgb'])} && D.pdifgb == {h(d['pdifgb'])};")
        w(f"    ok = ok && D.ncocon == {d['ncocon']} && D.ncovis == {d['ncovis']} && D.ncodif == {d['ncodif']};")
        for s in range(ns):
            for q in range(d["ncocon"]):
                w(f"    ok = ok && D.condco[{s}][{q}] == {h(d['condco'][s][q])};")
            for q in range(d["ncovis"]):
                w(f"    ok = ok && D.viscco[{s}][{q}] == {h(d['viscco'][s][q])};")
            for t in range(ns):
                w(f"    ok = ok && D.wilko1[{s}][{t}] == {h(d['wilko1'][s][t])} && D.wilko2[{s}][{t}] == {h(d['wilko2'][s][t])};")
                for q in range(d["ncodif"]):
                    w(f"    ok = ok && D.diffco[{s}][{t}][{q}] == {h(d['diffco'][s][t][q])};")
    w("    return ok;")
    w("  }")
    w("};")
    return "\n".join(o)


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "mech_gen.cuh")
    parts = ["// GENERATED by gen_mech.py from ../data/*.dat -- do not edit.",
             "// Straight-line thermochemistry policies (see gen_mech.py).",
             "#pragma once", "#include <cstdint>", '#include "senga_gpu.h"', "", "namespace senga {", "namespace gen {", ""]
    c1 = load_chem(os.path.join(DATA, "chem_1step.dat"))
    parts.append(gen("onestep", c1, None))
    ch2 = load_chem(os.path.join(DATA, "chem_h2.dat"))
    dh2 = load_diff(os.path.join(DATA, "diff_h2.dat"), ch2)
    parts.append(gen("h2", ch2, dh2))
    parts += ["", "}  // namespace gen", "}  // namespace senga", ""]
    with open(out, "w") as fh:
        fh.write("\n".join(parts))


if __name__ == "__main__":
    main()
