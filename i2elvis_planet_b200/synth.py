"""Seeded synthetic planetesimal instances for the marker step.

The reference builds its initial state with ``in2mart`` (in2mart.c:24-1486): grid
lines by accumulation (in2mart.c:130-133), a k x k marker lattice per cell laid out
cell-major (in2mart.c:155-182) and a random jitter (in2mart.c:187-197).  This module
builds the same kind of state from a counter-based generator (splitmix64 of
(seed, stream, index)), so every consumer -- the CUDA path, the oracle and the
compiled reference -- receives bit-identical inputs.

Workloads (square box L = 500 km, node layout ``m3 = m1*ynumy + m2``):

====== =========== ===== ====== ==========================================
name   nodes       k     steps  notes
====== =========== ===== ====== ==========================================
micro  21 x 21     4     2      tiny parity case
c1     101 x 101   4     1      CPU-runnable case
c2     401 x 401   4     10     FP64 and mixed
c3     1001 x 1001 6     10     8 extra stream-function modes, eta clipped
                                to [1e18, 1e24], random storage order
c5     201 x 201   4     20     adjoint case (8 mode amplitudes)
p6     601 x 601   6     10     c3 construction at profiling size
====== =========== ===== ====== ==========================================

The batched workload (64 instances with random sizes) is :func:`make_batch`.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

L_BOX = 500e3
NTYPES = 200
SEED_BASE = 20261203

# Per-type table names, in the order the C ABI's i2g_types struct and the
# reference harness file layout use (reference arrays headmart.c:128-132).
TYPE_TABLES = (
    "marknu", "markdh", "markdv", "markss", "markmm", "markll", "marka0", "marka1",
    "markb0", "markb1", "marke0", "marke1", "markro", "markaa", "markbb", "markcp",
    "markkt", "markht", "markkf", "markkp", "markn0", "markn1", "marks0", "marks1",
)
GRID_FIELDS = ("vx", "vy", "pr", "exx", "eyy", "exy", "sxx", "syy", "sxy", "ga", "mu")
NODE_OUT = ("ro", "nu", "nd", "et", "cp", "kt", "ht", "tk", "po")

SEC_PER_YEAR = 365.25 * 24 * 3600.0

# rock types of the synthetic planetesimal: air, silicate, iron
TYPE_AIR, TYPE_SIL, TYPE_FE = 0, 5, 7
ROCKS = {
    # type: (rho kg/m^3, eta Pa s, k W/m/K, Cp J/kg/K)
    TYPE_AIR: (1.0, 1e18, 3.0, 1000.0),
    TYPE_SIL: (3300.0, 1e20, 3.0, 1000.0),
    TYPE_FE: (7800.0, 1e19, 40.0, 800.0),
}


# ---------------------------------------------------------------- counter RNG
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64, copy=True)
    with np.errstate(over="ignore"):
        z += np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def rng_u64(seed: int, stream: int, n: int, offset: int = 0) -> np.ndarray:
    """n raw 64-bit draws for (seed, stream), counter-based (index = offset..offset+n-1)."""
    base = _splitmix64(np.array([(seed & 0xFFFFFFFF) | ((stream & 0xFFFF) << 32)], dtype=np.uint64))[0]
    idx = np.arange(offset, offset + n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _splitmix64(idx * np.uint64(0xD1B54A32D192ED03) + base)


def rng_uniform(seed: int, stream: int, n: int) -> np.ndarray:
    """Uniform doubles in [0, 1) with 53 random bits."""
    return (rng_u64(seed, stream, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def rng_normal(seed: int, stream: int, n: int) -> np.ndarray:
    """Standard normal draws (Box-Muller on two uniform streams)."""
    u1 = rng_uniform(seed, stream, n)
    u2 = rng_uniform(seed, stream + 1, n)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


def _erf(x: np.ndarray) -> np.ndarray:
    from scipy.special import erf
    return erf(x)


# ---------------------------------------------------------------- instance
@dataclass
class Instance:
    """One planetesimal: grid, node fields, markers, per-type tables and flags."""
    name: str
    xnumx: int
    ynumy: int
    xsize: float
    ysize: float
    gx: np.ndarray
    gy: np.ndarray
    grid: dict               # GRID_FIELDS -> float64[nodenum]
    nodes: dict              # NODE_OUT -> float64[nodenum] (initial node state)
    x: np.ndarray
    y: np.ndarray
    T: np.ndarray
    eta: np.ndarray
    mtype: np.ndarray        # int8
    hi: np.ndarray
    por: np.ndarray
    tmax: np.ndarray
    types: dict              # TYPE_TABLES -> float64[200]
    markim: np.ndarray       # int64[200]
    timestep: float
    timesum: float
    nsteps: int
    mnumx: int
    mnumy: int
    flags: dict = field(default_factory=dict)
    scal: dict = field(default_factory=dict)
    modes: np.ndarray | None = None      # (nmodes, 2) integer wavenumbers
    amps: np.ndarray | None = None       # (nmodes,) stream-function amplitudes
    mode_vx: np.ndarray | None = None    # (nmodes, nodenum) unit-amplitude vx per mode
    mode_vy: np.ndarray | None = None
    td: dict | None = None               # densimod 2 P-T table (td_table)
    # marker fields the output file carries that the marker step does not read
    # (headmart.c:119-127): grain size, accretion time, magnetisation state and time
    gr: np.ndarray | None = None
    acc: np.ndarray | None = None
    mg_old: np.ndarray | None = None     # int8
    mg_time: np.ndarray | None = None

    @property
    def nodenum(self) -> int:
        return self.xnumx * self.ynumy

    @property
    def marknum(self) -> int:
        return int(self.x.shape[0])

    def copy(self) -> "Instance":
        import copy as _c
        return _c.deepcopy(self)


def default_flags() -> dict:
    """Hot-path switches of mode.t3c (mode.t3c:6010-6031) used by every workload."""
    return dict(markmod=2, outgrid=2, intermod=0, intermod1=0, gridmod=1, densimod=0,
                viscmod=1, dynamo=0)


def default_scal() -> dict:
    return dict(nubeg=1e17, nuend=1e26, nucontr=1e18, tmp_ambient=150.0, M_init=0.0, M_acc=0.0,
                core_form_time=1e30, k_cutoff=1.0e6, al2627_init=5.25e-5, fe6056_init=1.15e-8,
                relax_time=0.010, por_init=0.0, eps21=0.0, eps50=0.0, eps52=0.0)


def default_types() -> tuple[dict, np.ndarray]:
    t = {k: np.zeros(NTYPES) for k in TYPE_TABLES}
    t["marknu"][:] = 1e20
    t["markmm"][:] = 1.0
    t["markn0"][:] = 1e17
    t["markn1"][:] = 1e26
    t["markro"][:] = 1.0
    t["markcp"][:] = 1000.0
    t["markkt"][:] = 3.0
    for ty, (rho, eta, k, cp) in ROCKS.items():
        t["markro"][ty] = rho
        t["marknu"][ty] = eta
        t["markkt"][ty] = k
        t["markcp"][ty] = cp
    return t, np.zeros(NTYPES, dtype=np.int64)


def td_table(seed: int, tknum: int = 350, pbnum: int = 350, si_melting: int = 1, fe_melting: int = 0,
             ice_melting: int = 1) -> dict:
    """A seeded stand-in for the thermodynamic table loadmart.c:116-209 reads from
    "mars_mantle" (database 0) and "mars_crust" (database 1), on the reference's P-T
    grid (loadmart.c:117-122): density (g/cm^3) with thermal expansion and
    compression, enthalpy (kcal/kg) with a heat capacity of 1200 (mantle) and 1100
    (crust) J/kg/K and a V(1 - alpha T) pressure term, each with a small seeded
    perturbation per node.  Layout td[tk][pb][db][k] of headmart.c:137 (k = 0
    density, 1 enthalpy; 2..4 unused, zero)."""
    tkmin, pbmin = 500.005, 1000.5
    tkstp = (5000.0 - tkmin) / (tknum - 1)
    pbstp = (500000.0 - pbmin) / (pbnum - 1)
    tk = tkmin + tkstp * np.arange(tknum)[:, None]
    pb = pbmin + pbstp * np.arange(pbnum)[None, :]
    td = np.zeros((tknum, pbnum, 2, 5))
    for db, (rho0, cp, alpha, kbar) in enumerate(((3.30, 1200.0, 3.0e-5, 1.3e6), (2.90, 1100.0, 3.5e-5, 0.9e6))):
        u = rng_uniform(seed, 10 + db, tknum * pbnum).reshape(tknum, pbnum) - 0.5
        v = rng_uniform(seed, 20 + db, tknum * pbnum).reshape(tknum, pbnum) - 0.5
        rho = rho0 * (1.0 - alpha * (tk - 298.15)) * (1.0 + pb / kbar) * (1.0 + 2e-4 * u)
        h = (cp * tk + 1e5 * pb / (rho0 * 1000.0) * (1.0 - alpha * tk)) / 4183.7
        td[:, :, db, 0] = rho
        td[:, :, db, 1] = h * (1.0 + 2e-5 * v)
    return dict(td=td, tknum=tknum, pbnum=pbnum, tkmin=tkmin, pbmin=pbmin, tkstp=tkstp, pbstp=pbstp,
                si_melting=si_melting, fe_melting=fe_melting, ice_melting=ice_melting)


def grid_lines(n: int, size: float) -> np.ndarray:
    """Grid lines by accumulation, as in2mart.c:130-133 builds them."""
    g = np.empty(n)
    step = size / (n - 1)
    acc = 0.0
    g[0] = 0.0
    for i in range(1, n):
        acc = acc + step
        g[i] = acc
    return g


def stream_velocity(gx, gy, modes, amps):
    """Discretely divergence-free staggered velocity from psi = sum a sin(p pi x/L) sin(q pi y/L).

    vx[i,j] = (psi[i,j+1]-psi[i,j])/dy sits at (gx[i], (gy[j]+gy[j+1])/2);
    vy[i,j] = -(psi[i+1,j]-psi[i,j])/dx sits at ((gx[i]+gx[i+1])/2, gy[j]).
    Returns per-mode unit-amplitude fields (nmodes, nx*ny) for vx and vy.
    """
    nx, ny = gx.size, gy.size
    Lx, Ly = gx[-1] - gx[0], gy[-1] - gy[0]
    mvx = np.zeros((len(modes), nx, ny))
    mvy = np.zeros((len(modes), nx, ny))
    for m, (p, q) in enumerate(modes):
        psi = np.outer(np.sin(p * np.pi * gx / Lx), np.sin(q * np.pi * gy / Ly))
        dy = np.diff(gy)[None, :]
        dx = np.diff(gx)[:, None]
        mvx[m, :, :-1] = (psi[:, 1:] - psi[:, :-1]) / dy
        mvy[m, :-1, :] = -(psi[1:, :] - psi[:-1, :]) / dx
    return mvx.reshape(len(modes), -1), mvy.reshape(len(modes), -1)


def make_instance(name: str, n: int, k: int, nsteps: int, seed: int, *, r_disk: float = 200e3,
                  vmax: float = 1e-9, extra_modes: int = 0, eta_clip=None, permute: bool = False,
                  delta: float | None = None, sigma_dec: float = 1.0,
                  mode_list=None, amps=None) -> Instance:
    L = L_BOX
    gx = grid_lines(n, L)
    gy = grid_lines(n, L)
    dxc = L / (n - 1)
    # ---- markers: k x k per cell at sub-cell centres, cell-major (in2mart.c:155-182)
    ncell = (n - 1) * (n - 1)
    m1 = np.repeat(np.arange(n - 1), (n - 1) * k * k)
    m2 = np.tile(np.repeat(np.arange(n - 1), k * k), n - 1)
    a = np.tile(np.repeat(np.arange(k), k), ncell)
    b = np.tile(np.arange(k), ncell * k)
    nm = ncell * k * k
    x = gx[m1] + (a + 0.5) * (dxc / k)
    y = gy[m2] + (b + 0.5) * (dxc / k)
    # jitter: uniform in [-0.5, 0.5] marker spacing per axis (in2mart.c:187-197 draws a 201-level rand())
    x = x + (rng_uniform(seed, 1, nm) - 0.5) * (dxc / k)
    y = y + (rng_uniform(seed, 2, nm) - 0.5) * (dxc / k)
    r = np.hypot(x - L / 2, y - L / 2)
    mtype = np.where(r > r_disk, TYPE_AIR, TYPE_SIL).astype(np.int8)
    iron = (rng_uniform(seed, 3, nm) < 0.2) & (mtype == TYPE_SIL)
    mtype[iron] = TYPE_FE
    eta0 = np.array([ROCKS[int(t)][1] if int(t) in ROCKS else 1e20 for t in range(NTYPES)])
    eta = eta0[mtype.astype(np.int64)] * 10.0 ** (sigma_dec * rng_normal(seed, 4, nm))
    if eta_clip is not None:
        eta = np.clip(eta, eta_clip[0], eta_clip[1])
    dlt = delta if delta is not None else r_disk / 2
    T = 150.0 + 1650.0 * _erf(np.maximum(0.0, r_disk - r) / dlt)
    if permute:
        perm = np.argsort(rng_u64(seed, 9, nm), kind="stable")
        x, y, T, eta, mtype = x[perm], y[perm], T[perm], eta[perm], mtype[perm]
    # ---- velocity from stream-function modes
    if mode_list is None:
        modes = [(1, 1)]
        u = rng_uniform(seed, 5, 3 * max(extra_modes, 1))
        for j in range(extra_modes):
            modes.append((1 + int(u[3 * j] * 8), 1 + int(u[3 * j + 1] * 8)))
        if amps is None:
            amps = [1.0] + [(0.3 if u[3 * j + 2] < 0.5 else -0.3) for j in range(extra_modes)]
    else:
        modes = list(mode_list)
    modes = np.asarray(modes, dtype=np.int64)
    amps = np.asarray(amps, dtype=np.float64)
    mvx, mvy = stream_velocity(gx, gy, modes, amps)
    vx = amps @ mvx
    vy = amps @ mvy
    scale = vmax / max(np.abs(vx).max(), np.abs(vy).max())
    amps = amps * scale
    vx = vx * scale
    vy = vy * scale
    # ---- pressure: seeded smooth field at cell centres (index m1>=1, m2>=1)
    ph = rng_uniform(seed, 6, 2) * 2 * np.pi
    xc = np.concatenate([[0.0], 0.5 * (gx[1:] + gx[:-1])])
    yc = np.concatenate([[0.0], 0.5 * (gy[1:] + gy[:-1])])
    pr = 1e8 * (1.0 + 0.5 * np.outer(np.sin(2 * np.pi * xc / L + ph[0]), np.cos(2 * np.pi * yc / L + ph[1])))
    pr[0, :] = 0.0
    pr[:, 0] = 0.0
    nn = n * n
    grid = {f: np.zeros(nn) for f in GRID_FIELDS}
    grid["vx"] = vx.copy()
    grid["vy"] = vy.copy()
    grid["pr"] = pr.reshape(-1).copy()
    nodes = {f: np.zeros(nn) for f in NODE_OUT}
    types, markim = default_types()
    inst = Instance(
        name=name, xnumx=n, ynumy=n, xsize=L, ysize=L, gx=gx, gy=gy,
        grid=grid, nodes=nodes, x=x, y=y, T=T, eta=eta, mtype=mtype,
        hi=np.zeros(nm), por=np.zeros(nm), tmax=T.copy(), types=types, markim=markim,
        timestep=0.5 * dxc / vmax, timesum=1.0e6 * SEC_PER_YEAR, nsteps=nsteps, mnumx=k, mnumy=k,
        flags=default_flags(), scal=default_scal(), modes=modes, amps=amps, mode_vx=mvx, mode_vy=mvy)
    return inst


CONFIGS = {
    "micro": dict(n=21, k=4, nsteps=2, idx=9),
    "c1": dict(n=101, k=4, nsteps=1, idx=1),
    "c2": dict(n=401, k=4, nsteps=10, idx=2),
    "c3": dict(n=1001, k=6, nsteps=10, idx=3, extra_modes=8, eta_clip=(1e18, 1e24), permute=True),
    "c5": dict(n=201, k=4, nsteps=20, idx=5, extra_modes=7),
    # profiling case: the c3 construction on a 601x601 grid (12.96M markers, ~1.3 GB)
    "p6": dict(n=601, k=6, nsteps=10, idx=6, extra_modes=8, eta_clip=(1e18, 1e24), permute=True),
}


def make_config(name: str, instance: int = 0, **over) -> Instance:
    """Build one of the named workloads; seed = 20261203 + 1000*config + instance."""
    c = dict(CONFIGS[name])
    c.update(over)
    idx = c.pop("idx")
    seed = SEED_BASE + 1000 * idx + instance
    return make_instance(name, seed=seed, **c)


def make_batch(ninst: int = 64, seed_instance0: int = 0, nmin: int = 101, nmax: int = 401,
               nsteps: int = 10) -> list[Instance]:
    """Batched workload: grids U{nmin..nmax}, disk radius U[50,250] km, k U{3..6},
    vmax log-uniform in [1e-10, 1e-8], temperature width per instance."""
    out = []
    for i in range(ninst):
        seed = SEED_BASE + 1000 * 4 + seed_instance0 + i
        u = rng_uniform(seed, 7, 5)
        n = nmin + int(u[0] * (nmax - nmin + 1))
        r_disk = 50e3 + u[1] * 200e3
        k = 3 + int(u[2] * 4)
        vmax = 10.0 ** (-10.0 + 2.0 * u[3])
        delta = r_disk * (0.25 + 0.5 * u[4])
        out.append(make_instance(f"b{i}", n=n, k=k, nsteps=nsteps, seed=seed, r_disk=r_disk, vmax=vmax,
                                 delta=delta, extra_modes=2))
    return out


def subset(inst: Instance, idx: np.ndarray) -> Instance:
    """The same instance restricted to the markers ``idx`` (grid unchanged)."""
    s = inst.copy()
    for f in ("x", "y", "T", "eta", "mtype", "hi", "por", "tmax"):
        setattr(s, f, np.ascontiguousarray(getattr(inst, f)[idx]))
    return s


def describe(inst: Instance) -> dict:
    return {"workload": inst.name, "nodes": f"{inst.xnumx}x{inst.ynumy}", "markers": inst.marknum,
            "markers_per_cell": f"{inst.mnumx}x{inst.mnumy}", "steps": inst.nsteps,
            "dt_s": inst.timestep}


__all__ = ["Instance", "make_config", "make_batch", "make_instance", "subset", "CONFIGS",
           "TYPE_TABLES", "GRID_FIELDS", "NODE_OUT", "rng_uniform", "rng_normal", "rng_u64",
           "grid_lines", "stream_velocity", "describe"]


def thermal_fields(inst: Instance, seed: int = 7, fluid_frac: float = 0.0, cold_frac: float = 0.0,
                   dT: float = 40.0) -> dict:
    """Node fields around one thermal solve, for the marker temperature update of
    titerate() (heatmart.c:514-697): the node temperature before the solve (set as
    inst.nodes['tk']) and after it ('tk_new', a smooth change of about dT kelvin),
    the node conductivity, density and heat capacity the diffusion term reads,
    and radiogenic heat (the reference's time-step limit needs a nonzero rate).
    fluid_frac of the rock markers become fluid types (50 + type: the update sets
    their T to the new node T) and cold_frac get T = 0 (the update resets them to
    the old node T first).  Modifies inst in place."""
    gx, gy = np.meshgrid(inst.gx, inst.gy, indexing="ij")
    X, Y = gx / inst.xsize, gy / inst.ysize
    tk_old = 300.0 + 900.0 * X * (1.0 - X) * 4.0 * np.sin(np.pi * Y) + 50.0 * np.cos(3.0 * np.pi * X * Y)
    tk_new = tk_old + dT * (np.sin(2.0 * np.pi * X + 0.3) * np.cos(np.pi * Y) + 0.25)
    inst.nodes["tk"] = tk_old.reshape(-1).copy()
    inst.nodes["kt"] = (2.5 + 1.5 * X * Y).reshape(-1)
    inst.nodes["ro"] = (3000.0 + 800.0 * Y).reshape(-1)
    inst.nodes["cp"] = (1000.0 + 200.0 * X).reshape(-1)
    inst.nodes["ht"] = np.full(inst.nodenum, 1e-8)
    u = rng_uniform(seed, 1, inst.marknum)
    rock = (inst.mtype > 1) & (inst.mtype < 50)
    inst.mtype = inst.mtype.copy()
    inst.mtype[rock & (u < fluid_frac)] += 50
    inst.T = inst.T.copy()
    inst.T[(inst.mtype < 50) & (u >= fluid_frac) & (u < fluid_frac + cold_frac)] = 0.0
    return {"tk_old": inst.nodes["tk"].copy(), "tk_new": tk_new.reshape(-1)}


def with_table(i: Instance, hirschmann: bool = False) -> Instance:
    """densimod 2: the P-T table path (tdbasecalc/meltpart1, markmart.c:2068-2652)
    on a seeded table.  Silicate and crust markers across their solidus, wet
    planetesimal markers across the water-ice melting range, molten types flipping
    back, and the molten-rock conductivity reading the melt fraction the previous
    table marker left (markmart.c:287, 509-560).  Herzberg solidus and ice melting,
    or (hirschmann) the Hirschmann solidus without ice and every second marker."""
    i.flags["densimod"] = 2
    i.td = td_table(4242, si_melting=0 if hirschmann else 1, ice_melting=0 if hirschmann else 1)
    u = rng_uniform(779, 1, i.marknum)
    w = rng_uniform(779, 2, i.marknum)
    sil = i.mtype == 5
    for lo, hi, t in ((0.0, 0.25, 6), (0.25, 0.35, 11), (0.35, 0.40, 12), (0.40, 0.55, 25),
                      (0.55, 0.62, 26), (0.62, 0.68, 31), (0.68, 0.72, 32)):
        i.mtype[sil & (u >= lo) & (u < hi)] = t
    wet = (i.mtype == 6) & (w < 0.4)
    i.T[wet] = 262.0 + 30.0 * rng_uniform(779, 3, int(wet.sum()))
    T = i.types
    for t in (5, 6, 11, 12, 25, 26, 31, 32):
        T["markro"][t] = 3300.0 if t % 20 in (5, 6) else 2900.0
        T["markbb"][t] = 3e-5
        T["markaa"][t] = 2e-5
        T["markkt"][t] = 3.0 if t < 20 else 2.0
        T["markkf"][t] = 150.0
        T["markkp"][t] = 2e-6
        T["marknu"][t] = 1e20 if t < 20 else 1e2
        T["markn0"][t] = 1e17 if t < 20 else 10.0
    # the last table marker partly molten: a melt state that carries into the next step
    last = np.nonzero(i.mtype != 0)[0][-1]
    i.mtype[last] = 25
    i.T[last] = 1700.0
    i.grid["ga"] = np.full(i.nodenum, 0.08)
    i.scal["core_form_time"] = 0.0
    i.scal["eps21"] = 0.5
    if hirschmann:
        i.flags["gridmod"] = 2
    return i
