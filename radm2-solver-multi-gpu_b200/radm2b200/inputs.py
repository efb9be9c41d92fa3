"""Seeded synthetic RADM2 cell inputs in the reference's per-cell layout.

The reference reads its fields from WRF text dumps that are not shipped
(mgpu.cu:343-417) and converts them per cell in dev_convert (mgpu.cu:513-646)
into VAR[cell][59] (molec/cm^3), FIX[cell][2] = {H2O, M}, TEMP[cell],
RC_N2O5[cell] and JV[cell][28].  This module produces those same arrays from
seeded distributions instead.  Every value is a pure function of
(seed, cell index, field), through a counter-based hash, so any subset of cells
is reproducible on its own and the CPU oracle and the GPU see identical inputs.

Workloads (the distributions are stated in the repository's baseline notes):
  "plain"   4,096 / 1,048,576 cells: T U(260,310) K, p U(500,1013) hPa,
            O3 20-80 ppb, NO+NO2 0.1-50 ppb, CO 80-300 ppb, VOCs 0.01-10 ppb,
            radicals 1e-6-1e-2 ppt (log-uniform), SZA U(0,80) deg, night_frac of
            cells with J = 0.
  "mixed"   4,194,304 cells: 20% urban (NOx 20-200 ppb), 40% remote clean
            (NOx 0.02-1 ppb), 40% night (NOx 0.1-50 ppb, J = 0), T U(220,310) K.
"""
import numpy as np

NVAR, NFIX, NPH = 59, 2, 28

# Physical constants of the conversion in mgpu.cu:29-43.
NAVOGADRO = 6.022e23
MW_AIR = 28.97
MW_H2O = 2 * 1.0079 + 15.9994
DENS2CON_A = 1.0e-3 * (1.0 / MW_AIR) * NAVOGADRO
DENS2CON_W = 1.0e-3 * (1.0 / MW_H2O) * NAVOGADRO
K_BOLTZMANN = 1.380649e-23

SPECIES = ["SULF", "ORA1", "ORA2", "CO2", "SO2", "ETH", "O1D", "HC5", "HC8", "TOL", "XYL", "TPAN", "HONO",
           "H2O2", "N2O5", "HC3", "CH4", "PAA", "O3P", "HNO4", "OP1", "CSL", "PAN", "OL2", "HNO3", "CO", "ISO",
           "OLT", "OLI", "DCB", "GLY", "XNO2", "KET", "MGLY", "TOLP", "XYLP", "OLTP", "OLN", "XO2", "OL2P",
           "HC5P", "OP2", "HCHO", "HC8P", "TCO3", "O3", "ONIT", "ALD", "OLIP", "KETP", "HO2", "MO2", "OH",
           "NO3", "ACO3", "HC3P", "ETHP", "NO", "NO2"]
IDX = {n: i for i, n in enumerate(SPECIES)}

VOCS = ["ETH", "HC3", "HC5", "HC8", "OL2", "OLT", "OLI", "ISO", "TOL", "XYL", "CSL", "HCHO", "ALD", "KET",
        "GLY", "MGLY", "DCB"]
RADICALS = ["O1D", "O3P", "OH", "HO2", "NO3", "MO2", "ACO3", "ETHP", "HC3P", "HC5P", "HC8P", "OL2P", "OLTP",
            "OLIP", "TOLP", "XYLP", "KETP", "TCO3", "XO2", "XNO2", "OLN"]
RESERVOIRS = ["SULF", "ORA1", "ORA2", "SO2", "TPAN", "HONO", "H2O2", "N2O5", "PAA", "HNO4", "OP1", "PAN",
              "HNO3", "ONIT", "OP2"]
# Mixing-ratio ranges in ppb (log-uniform).
RANGES = {"O3": (20.0, 80.0), "CO": (80.0, 300.0), "CH4": (1700.0, 1900.0), "CO2": (380.0e3, 420.0e3)}
for _n in VOCS + RESERVOIRS:
    RANGES[_n] = (0.01, 10.0)
for _n in RADICALS:
    RANGES[_n] = (1.0e-9, 1.0e-5)  # 1e-6 .. 1e-2 ppt
assert set(RANGES) | {"NO", "NO2"} == set(SPECIES)

# Clear-sky photolysis rates at SZA = 0 (1/s) and cos(SZA) exponents for the 28
# reference photolysis slots (mgpu.cu:52-79); J = J0 cos(SZA)^n by day, 0 at night.
J0 = [3.0e-5, 4.5e-4, 9.0e-3, 2.2e-2, 1.8e-1, 2.0e-3, 7.0e-7, 5.0e-6, 8.0e-6, 3.0e-5, 4.5e-5, 5.0e-6, 6.0e-7,
      1.5e-6, 3.0e-5, 1.4e-4, 1.0e-4, 6.0e-6, 2.0e-6, 1.0e-6, 4.0e-5, 3.0e-6, 3.0e-5, 1.0e-11, 3.0e-7, 5.0e-7,
      1.0e-4, 4.0e-6]
JN = [2.0, 0.5, 0.4, 0.25, 0.25, 0.4, 1.2, 0.9, 0.8, 0.8, 0.7, 1.0, 1.3, 1.1, 0.6, 0.6, 0.6, 0.8, 0.9, 1.2, 0.6,
      0.9, 0.8, 1.0, 1.2, 1.2, 0.6, 0.9]

# Hash field identifiers.
F_T, F_P, F_RH, F_SZA, F_CLASS, F_NOFRAC, F_NOX = range(7)
F_SPECIES0 = 16

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _mix(x):
    """splitmix64 finaliser on uint64 arrays (wrapping arithmetic)."""
    x = x ^ (x >> np.uint64(30))
    x = x * np.uint64(0xBF58476D1CE4E5B9)
    x = x ^ (x >> np.uint64(27))
    x = x * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def uniform(seed, cells, field):
    """U[0,1) per (seed, cell, field); cells is a uint64 array of global cell indices."""
    with np.errstate(over="ignore"):
        k = (np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)) ^ (np.uint64(field + 1) * np.uint64(0xD1B54A32D192ED03))
        x = _mix(cells * np.uint64(0x8CB92BA72F3D8DD7) + _mix(np.full(1, k, dtype=np.uint64))[0])
    return (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _logu(u, lo, hi):
    return np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))


def make_cells(ncell, seed, workload="plain", night_frac=0.3, first_cell=0):
    """Return dict VAR, FIX, TEMP, RC_N2O5, JV (reference layout) and cls (0 day, 1 urban, 2 remote, 3 night)."""
    cells = np.arange(first_cell, first_cell + ncell, dtype=np.uint64)
    u = lambda f: uniform(seed, cells, f)  # noqa: E731
    ucls = u(F_CLASS)
    if workload == "plain":
        T = 260.0 + 50.0 * u(F_T)
        cls = np.where(ucls < night_frac, 3, 0).astype(np.int32)
        nox = _logu(u(F_NOX), 0.1, 50.0)
    elif workload == "mixed":
        T = 220.0 + 90.0 * u(F_T)
        cls = np.where(ucls < 0.2, 1, np.where(ucls < 0.6, 2, 3)).astype(np.int32)
        unox = u(F_NOX)
        nox = np.where(cls == 1, _logu(unox, 20.0, 200.0),
                       np.where(cls == 2, _logu(unox, 0.02, 1.0), _logu(unox, 0.1, 50.0)))
    else:
        raise ValueError("unknown workload %r" % workload)
    p_hpa = 500.0 + 513.0 * u(F_P)
    p_pa = 100.0 * p_hpa
    M = p_pa / (K_BOLTZMANN * T) * 1.0e-6  # molec/cm^3
    rho = M / DENS2CON_A                     # kg/m^3, inverse of mgpu.cu:538
    # Water from relative humidity with the reference's saturation formula (mgpu.cu:548-550).
    rh = 0.2 + 0.7 * u(F_RH)
    es = 1000.0 * 0.6112 * np.exp(17.67 * (T - 273.15) / (T - 29.65))
    qvs = es / (p_pa - es)
    H2O = DENS2CON_W * (rh * qvs) * rho
    rc_n2o5 = 1.0 / (3.6e4 * np.exp(-np.power(rh / 0.28, 2.8) + 300.0))  # mgpu.cu:552

    ppb = M * 1.0e-9
    VAR = np.empty((ncell, NVAR), dtype=np.float64)
    for name, (lo, hi) in RANGES.items():
        i = IDX[name]
        VAR[:, i] = _logu(u(F_SPECIES0 + i), lo, hi) * ppb
    fno = 0.1 + 0.4 * u(F_NOFRAC)
    VAR[:, IDX["NO"]] = fno * nox * ppb
    VAR[:, IDX["NO2"]] = (1.0 - fno) * nox * ppb

    sza = np.deg2rad(80.0 * u(F_SZA))
    mu = np.cos(sza)
    JV = np.power(mu[:, None], np.asarray(JN)[None, :]) * np.asarray(J0)[None, :]
    JV[cls == 3, :] = 0.0
    FIX = np.stack([H2O, M], axis=1)
    return {"VAR": np.ascontiguousarray(VAR), "FIX": np.ascontiguousarray(FIX), "TEMP": T,
            "RC_N2O5": rc_n2o5, "JV": np.ascontiguousarray(JV), "cls": cls}


# Named workloads: (ncell, seed, workload, night_frac, nsplit).
WORKLOADS = {
    "plain-4k": (4096, 0, "plain", 0.0, 1),
    "plain-1m": (1048576, 1, "plain", 0.3, 6),
    "mixed-4m": (4194304, 2, "mixed", 0.4, 24),
    "mixed-4m-eval": (4194304, 3, "mixed", 0.4, 24),
}


# WRF field sets of the reference's conversion step (mgpu.cu:255-260, 477-484): chem 82,
# rad 29, ph 28, phy 3, moist 6 fields, each [nj][nk][ni] = [48][20][48] there.
WRF_NFIELDS = {"chem": 82, "rad": 29, "ph": 28, "phy": 3, "moist": 6}


def make_wrf_fields(seed, ni=48, nk=20, nj=48, neg_frac=0.01):
    """Seeded WRF-like fields, field-major with i fastest: [nfield][nj][nk][ni].

    phy: 0 pressure U(50, 101.3) kPa in Pa, 1 temperature U(220, 310) K, 2 air density
    p / (287.05 T); moist 1: water vapour 1e-5..2e-2 kg/kg (log-uniform, other moist
    fields the same); chem / rad: mixing ratios 1e-9..1e-1 ppmV log-uniform, a fraction
    neg_frac slightly negative (WRF advection undershoots, clamped by the conversion);
    ph: photolysis rates per minute, J0 * 60 * cos(SZA)^n with SZA U(0, 90) deg per column.
    Every value is a pure function of (seed, field, point)."""
    n = ni * nk * nj
    pts = np.arange(n, dtype=np.uint64)
    col = (pts % np.uint64(ni)) + np.uint64(ni) * (pts // np.uint64(ni * nk))  # (i, j): one column

    def u(fid, idx=pts):
        return uniform(seed, idx, 1000 + fid)

    pres = 100.0 * (500.0 + 513.0 * u(1))
    temp = 220.0 + 90.0 * u(2)
    rho = pres / (287.05 * temp)
    phy = np.stack([pres, temp, rho]).reshape(3, nj, nk, ni)
    qv = _logu(u(3), 1.0e-5, 2.0e-2)
    moist = np.stack([qv] * WRF_NFIELDS["moist"]).reshape(-1, nj, nk, ni)

    def mixing(fid):
        x = _logu(u(fid), 1.0e-9, 1.0e-1)
        return np.where(u(fid + 5000) < neg_frac, -0.1 * x, x)

    chem = np.stack([mixing(100 + f) for f in range(WRF_NFIELDS["chem"])]).reshape(-1, nj, nk, ni)
    rad = np.stack([mixing(300 + f) for f in range(WRF_NFIELDS["rad"])]).reshape(-1, nj, nk, ni)
    mu = np.cos(np.deg2rad(90.0 * u(4, col)))
    ph = np.stack([60.0 * J0[k] * np.power(mu, JN[k]) for k in range(NPH)]).reshape(NPH, nj, nk, ni)
    return {"ph": ph, "chem": chem, "rad": rad, "phy": phy, "moist": moist}
