"""Writes the golden fixtures of tests/golden/ from the reference's own test data.

    python tests/golden/make_golden.py /path/to/reference

crossing_jets_{MK,IG,AG}.npz: the fields the reference's own binary wrote after 5000
iterations of its crossing-jets validation cases (test/Doisneau/<closure>/reference/
part-field.tec), every cell-centred variable as float64 in (j, i) order, plus the
boundary table of the case (test/Doisneau/<closure>/INPUT/part-bc.txt) reduced to one
row per record: b i j k f code [alpha] -- so that the test can check the case it builds
against the reference's inputs before comparing fields.

chimera_IG.npz: the reference's overlapping-grid variant of the IG case (test/Doisneau/IG-chimera):
the node coordinates of its two blocks (tensor-product meshes: x, y, z per block, MESH/mesh.tec), its
boundary table (INPUT/part-bc.txt: b i j k f code per row, the six inlet reals of each 402 row, and
the donors of each 102 row: counts per ghost layer, then b i j k and weight per donor) and the bulk
density the reference's binary wrote after 5000 iterations (reference/part-field.tec), per block in
(j, i) order.

correlations.npz: the drag coefficient and the Nusselt number of every correlation the reference
offers, from the reference's own Python restatement of them (test/verification/common.py:
drag_coefficient, nusselt), on a grid of Reynolds, Mach, temperature-ratio and Prandtl numbers.

evaporation.npz: from the reference's own Python restatement of the published correlations
(test/verification/F-evaporation/run.py: slope, coupled, surface_state), at the conditions of its parts
1-4: the d-squared slopes K of the five evaporation models at 300 K and at the boiling clamp (380 K),
the bulk density of the Langmuir-Knudsen case at both, and the RK4 bulk density and temperature of the
d2-law, ASM and TC droplets with the temperature released (cp 4180) after 0.05 s.

ag_riemann.npz: the reference's Riemann problems of the anisotropic Gaussian closure. For each Berthon case
(test/Berthon/{SCS,RCS,RCR,SCS-hlle}): the initial cell states (INPUT/part-ic.tec, the 12 primitives
along x), the time threshold (input.ini), the L1 tolerance its verify.py passes and the tabulated exact
wave pattern (Results/<case>/<case>_exact.tec: abscissae and values of the six piecewise-linear profiles,
density, u, v, P11, P22 and det P, in that order). For the anisotropic Sod tube (test/Riemann/AG): the
constants of make_case.py (grid, states, drop radius and density), the time threshold and the gates of
its verify.py.

restart_counters.npz: the counters the reference's binary stored beside its crossing-jets solutions
(test/Doisneau/{MK,IG,AG,IG-chimera}/reference/part-field.tec, DATASETAUXDATA): CYCLE, ICE_ITERATION,
ICE_RES_REFERENCE (the first non-zero density residual of the run: the unit of res-threshold), per case.

tecplot_sample.npz: the text of the reference's solution files (test/Doisneau/{MK,IG,AG}/reference/
part-field.tec, written by its Tecplot writer): per case the two header lines, the data set auxiliary
data lines of the restart counters, and a sample of the value lines (every 97th, and the first 200
negative ones), as strings, with their positions among the value lines.

The reference is read here, in this container; the fixtures travel, the reference does not.
"""
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def read_field(path):
    text = Path(path).read_text().split("\n")
    zi = next(i for i, l in enumerate(text) if "ZONE" in l)
    g = lambda k: int(re.search(r"\b%s\s*=\s*(\d+)" % k, text[zi]).group(1))
    I, J, K = g("I"), g("J"), g("K")
    vals = np.array([float(t) for l in text[zi + 1:] if not l.lstrip().startswith("DATASETAUXDATA")
                     for t in l.split()])
    Nn, Nc = I * J * K, (I - 1) * (J - 1) * max(K - 1, 1)
    nv = (len(vals) - 3 * Nn) // Nc
    cells = vals[3 * Nn:3 * Nn + nv * Nc].reshape(nv, max(K - 1, 1), J - 1, I - 1)
    return cells[:, 0]                         # (nv, j, i) of the single k layer


def read_bc(path):
    rows = []
    lines = Path(path).read_text().split("\n")
    q = 0
    while q < len(lines):
        t = lines[q].split()
        q += 1
        if len(t) != 6:
            continue
        b, i, j, k, f, code = map(int, t)
        alpha = 0.0
        if 401 <= code <= 403:
            alpha = float(lines[q].split()[2])
            q += 1
        rows.append((b, i, j, k, f, code, alpha))
    return np.array(rows)


def tec_zones(path):
    """(I, J, K, values) of every zone of a Tecplot ASCII block-packed file."""
    lines = Path(path).read_text().split("\n")
    heads = [i for i, l in enumerate(lines) if re.match(r"\s*ZONE\b", l)]
    out = []
    for a, z in enumerate(heads):
        end = heads[a + 1] if a + 1 < len(heads) else len(lines)
        hdr, vals = lines[z], []
        for l in lines[z + 1:end]:
            if re.search(r"[A-DF-Za-df-z]", l):       # header continuation lines (I=, DATAPACKING=, ...)
                hdr += " " + l
                continue
            vals += [float(t) for t in l.split()]
        g = lambda k: int(re.search(r"\b%s\s*=\s*(\d+)" % k, hdr).group(1))
        out.append((g("I"), g("J"), g("K"), np.array(vals)))
    return out


def read_chimera_bc(path):
    """Rows b i j k f code; the six inlet reals of 402/401/403 rows; the donors of 102 rows."""
    lines = [l for l in Path(path).read_text().split("\n") if l.strip()]
    rows, pay, cn, don, wts = [], [], [], [], []
    q = 0
    while q < len(lines):
        b, i, j, k, f, code = map(int, lines[q].split())
        q += 1
        p6 = [0.0] * 6
        n12 = [0, 0]
        if 401 <= code <= 403:
            p6 = [float(t) for t in lines[q].split()[:6]]
            q += 1
        elif code in (101, 201):
            q += 1
        elif code == 102:
            n12 = [int(t) for t in lines[q].split()[:2]]
            q += 1
            for _ in range(sum(n12)):
                t = lines[q].split()
                don.append([int(x) for x in t[:4]]); wts.append(float(t[4]))
                q += 1
        rows.append((b, i, j, k, f, code)); pay.append(p6); cn.append(n12)
    return (np.array(rows, dtype=np.int32), np.array(pay), np.array(cn, dtype=np.int32),
            np.array(don, dtype=np.int32).reshape(-1, 4), np.array(wts))


def chimera(ref):
    case = ref / "test" / "Doisneau" / "IG-chimera"
    out = {}
    for b, (I, J, K, v) in enumerate(tec_zones(case / "MESH" / "mesh.tec"), start=1):
        N = I * J * K
        x, y, z = (v[a * N:(a + 1) * N].reshape(K, J, I) for a in range(3))
        assert np.all(x == x[:1, :1, :]) and np.all(y == y[:1, :, :1]) and np.all(z == z[:, :1, :1])
        out[f"x{b}"], out[f"y{b}"], out[f"z{b}"] = x[0, 0, :], y[0, :, 0], z[:, 0, 0]
    for b, (I, J, K, v) in enumerate(tec_zones(case / "reference" / "part-field.tec"), start=1):
        Nn, Nc = I * J * K, (I - 1) * (J - 1) * max(K - 1, 1)
        out[f"rho{b}"] = v[3 * Nn:3 * Nn + Nc].reshape(J - 1, I - 1)
    rows, pay, cn, don, wts = read_chimera_bc(case / "INPUT" / "part-bc.txt")
    out.update(bc=rows, inlet=pay, nchi=cn, donor=don, weight=wts)
    np.savez_compressed(HERE / "chimera_IG.npz", **out)
    print("chimera_IG", rows.shape, don.shape, out["rho1"].shape, out["rho2"].shape)


DRAG_LAWS = ["Newton", "Stokes", "Schlichting", "Schiller-Naumann", "Wen-Yu", "Putnam", "Clift-Gauvin",
             "Morsi-Alexander", "Carlson-Hoglund", "Henderson", "Crowe", "Hermsen"]
HEAT_LAWS = ["Stokes", "JAXA1", "JAXA2", "JAXA3", "JAXA4", "Ranz-Marshall", "Kavanau-Drake"]


def correlations(ref):
    import importlib.util
    spec = importlib.util.spec_from_file_location("ice_verification_common", ref / "test" / "verification" / "common.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    re_ = np.concatenate([np.logspace(-2, 5, 29), [999.0, 1000.0, 1001.0, 2e5, 3e5]])
    ma = np.array([0.05, 0.3, 0.8, 1.0, 1.2, 1.75, 2.5])
    tr = np.array([0.5, 1.0, 2.0])
    pr = np.array([0.7, 1.0])
    out = {"Re": re_, "Ma": ma, "Tr": tr, "Pr": pr, "G": np.array(1.4)}
    for law in DRAG_LAWS:
        out["cd_" + law] = np.array([[[mod.drag_coefficient(law, R, M, 1.4, T) for T in tr] for M in ma] for R in re_])
    for law in HEAT_LAWS:
        out["nu_" + law] = np.array([[[mod.nusselt(law, R, P, M) for M in ma] for P in pr] for R in re_])
    np.savez_compressed(HERE / "correlations.npz", **out)
    print("correlations", len(DRAG_LAWS), len(HEAT_LAWS), re_.size)


def evaporation(ref):
    import importlib.util
    sys.path.insert(0, str(ref / "test" / "verification"))
    spec = importlib.util.spec_from_file_location("ice_verification_f", ref / "test" / "verification" / "F-evaporation" / "run.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    models = list(mod.MODELS)
    k = np.array([mod.slope(m) for m in models])
    rho_lk, tp_lk = mod.coupled("CEM", 0.04, mod.CS_FROZEN, interface="LK")
    free = ["d2-law", "ASM", "TC"]
    hot = np.array([mod.coupled(m, 0.05, mod.CS_L) for m in free])            # (rho_p, T_p) per model
    t_boil = (1.0 - 0.9 ** (2.0 / 3.0)) * mod.D0 ** 2 / mod.slope("CEM", Tp=380.0)
    k_boil = np.array([mod.slope(m, Tp=380.0) for m in models])
    rho_lk_boil, _ = mod.coupled("CEM", t_boil, mod.CS_FROZEN, interface="LK", steps=4000, tp0=380.0)
    np.savez_compressed(HERE / "evaporation.npz", models=np.array(models), K=k, t_lk=np.array(0.04),
                        rho_lk=np.array(rho_lk), K_lk=np.array(mod.slope("CEM", interface="LK")),
                        free=np.array(free), hot=hot, t_boil=np.array(t_boil), K_boil=k_boil,
                        rho_lk_boil=np.array(rho_lk_boil))
    print("evaporation", dict(zip(models, k)), rho_lk, hot, t_boil)


BERTHON_ZONES = ("Density", "X Velocity", "Y Velocity", "XX Pressure", "YY Pressure", "Det Pressure")


def ag_riemann(ref):
    out = {}
    for case in ("SCS", "RCS", "RCR", "SCS-hlle"):
        d = ref / "test" / "Berthon" / case
        key = case.replace("-", "_")
        text = (d / "INPUT" / "part-ic.tec").read_text().split("\n")
        zi = next(i for i, l in enumerate(text) if "ZONE" in l)
        g = lambda k: int(re.search(r"\b%s\s*=\s*(\d+)" % k, text[zi]).group(1))
        I, J, K = g("I"), g("J"), g("K")
        vals = np.array([float(t) for l in text[zi + 1:] for t in l.split()])
        nn, nc = I * J * K, (I - 1) * (J - 1) * (K - 1)
        out[key + "_x"] = vals[:I]
        out[key + "_ic"] = vals[3 * nn:3 * nn + 12 * nc].reshape(12, K - 1, J - 1, I - 1)[:, 0, 0, :]
        ini = (d / "input.ini").read_text()
        out[key + "_t"] = np.array(float(re.search(r"time-threshold\s*=\s*([-+.\deE]+)", ini).group(1)))
        out[key + "_hlle"] = np.array("HLLE" in ini)
        out[key + "_tol"] = np.array(float(re.search(r"tol\s*=\s*([-+.\deE]+)", (d / "verify.py").read_text()).group(1)))
        src = case.split("-")[0]
        lines = (ref / "test" / "Berthon" / "Results" / src / f"{src}_exact.tec").read_text().split("\n")
        zones = {}
        q = 0
        while q < len(lines):
            m = re.search(r'ZONE\s+T\s*=\s*"([^"]+)"', lines[q])
            if not m:
                q += 1
                continue
            n = int(re.search(r"\bI\s*=\s*(\d+)", lines[q + 1]).group(1))
            q += 3
            v = []
            while len(v) < 2 * n:
                v += [float(t) for t in lines[q].split()]
                q += 1
            zones[m.group(1)] = np.array(v[:2 * n])
        for z, name in enumerate(BERTHON_ZONES):
            out[f"{key}_exact{z}"] = zones[name].reshape(2, -1)
    d = ref / "test" / "Riemann" / "AG"
    mc = (d / "make_case.py").read_text()
    for lhs, rhs in re.findall(r"^((?:NX|X0),[^=]*)=\s*(.*)$", mc, re.M):
        for name, v in zip(lhs.split(","), rhs.split(",")):
            out["sod_" + name.strip()] = np.array(float(v))
    ini = (d / "input.ini").read_text()
    out["sod_t"] = np.array(float(re.search(r"time-threshold\s*=\s*([-+.\deE]+)", ini).group(1)))
    gates = re.search(r"^NAME, GAMMA, T_END, L1_TOL, P11_MIN, PT_TOL, TV_TOL\s*=\s*(.*)$",
                      (d / "verify.py").read_text(), re.M).group(1).split(",")[1:]
    for name, v in zip(("GAMMA", "T_END", "L1_TOL", "P11_MIN", "PT_TOL", "TV_TOL"), gates):
        out["sod_" + name] = np.array(float(v))
    np.savez_compressed(HERE / "ag_riemann.npz", **out)
    print("ag_riemann", {k: v for k, v in out.items() if v.ndim == 0})


def restart_counters(ref):
    out = {}
    for case in ("MK", "IG", "AG", "IG-chimera"):
        text = (ref / "test" / "Doisneau" / case / "reference" / "part-field.tec").read_text()
        key = case.replace("-", "_")
        for name in ("CYCLE", "ICE_ITERATION", "ICE_RES_REFERENCE"):
            m = re.search(r'DATASETAUXDATA\s+%s\s*=\s*"([^"]+)"' % name, text)
            out[f"{key}_{name}"] = np.array(float(m.group(1)))
    np.savez_compressed(HERE / "restart_counters.npz", **out)
    print("restart_counters", {k: float(v) for k, v in out.items()})


def tecplot_sample(ref):
    out = {}
    for case in ("MK", "IG", "AG"):
        lines = (ref / "test" / "Doisneau" / case / "reference" / "part-field.tec").read_text().split("\n")
        head, body = lines[:2], [l for l in lines[2:] if l and not l.startswith("DATASETAUXDATA")]
        aux = [l for l in lines if l.startswith("DATASETAUXDATA")]
        idx = list(range(0, len(body), 97)) + [n for n, l in enumerate(body) if l.startswith("-")][:200]
        out[f"{case}_head"] = np.array(head)
        out[f"{case}_aux"] = np.array(aux)
        out[f"{case}_values"] = np.array([body[n] for n in idx])
        out[f"{case}_index"] = np.array(idx)
    np.savez_compressed(HERE / "tecplot_sample.npz", **out)
    print("tecplot_sample", {k: len(v) for k, v in out.items()})


def main(ref):
    ref = Path(ref)
    for cl in ("MK", "IG", "AG"):
        case = ref / "test" / "Doisneau" / cl
        field = read_field(case / "reference" / "part-field.tec")
        bc = read_bc(case / "INPUT" / "part-bc.txt")
        np.savez_compressed(HERE / f"crossing_jets_{cl}.npz", field=field, bc=bc)
        print(cl, field.shape, bc.shape)
    chimera(ref)
    correlations(ref)
    evaporation(ref)
    ag_riemann(ref)
    restart_counters(ref)
    tecplot_sample(ref)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference")
    main(sys.argv[1])
