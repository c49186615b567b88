"""Seeded synthetic systems of the benchmark shapes (no datasets needed).

Units are Ndyn's: eV, Angstrom, amu; time unit 10.18 fs; kB = 8.6173303e-5
eV/K.  Positions are fractional in [-0.5, 0.5) as read_model leaves them
(src/read_input.f90:378-380).  Velocities are Maxwell-Boltzmann at T with
the mean velocity removed, as normalVelocityDistribution does
(src/nd.f90:1598-1621), drawn from numpy's PCG64 with the given seed.

Every builder returns a dict:
    masses, pairs, typ, pos, box, vel, control (keyword args of
    Context.set_control), name
"""
import math

import numpy as np

KB = 8.6173303e-5

CU_MORSE = dict(masses=[63.546], pairs=[(1, 1, True, "morse", [6.0, 0.3429, 1.3588, 2.866])],
                a=3.615, skin=0.5)
AR_LJ = dict(masses=[39.948], pairs=[(1, 1, True, "LJ", [8.5125, 0.0104, 3.405])],
             a=5.71903, skin=1.0215)
# Buckingham parameter order on a Pairs line is rc A rho C (src/potentials.f90:114-117)
NACL_BUCK = dict(masses=[22.99, 35.45],
                 pairs=[(1, 1, True, "buck", [8.0, 1000.0, 0.30, 0.0]),
                        (2, 2, True, "buck", [8.0, 3000.0, 0.32, 20.0]),
                        (1, 2, True, "buck", [8.0, 1500.0, 0.31, 5.0])],
                 a=5.64, skin=-1.0)

FCC_BASIS = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
ROCKSALT_NA = FCC_BASIS
ROCKSALT_CL = FCC_BASIS + np.array([0.5, 0.0, 0.0])


def lattice(cells, a, basis):
    nx, ny, nz = cells
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"),
                 -1).reshape(-1, 1, 3)
    pts = (g + basis[None]).reshape(-1, 3)
    box = np.array([nx * a, ny * a, nz * a], np.float64)
    frac = pts / np.array([nx, ny, nz], np.float64) - 0.5
    return frac, box


def jitter(pos, box, amp, rng):
    if amp <= 0:
        return pos
    return pos + rng.uniform(-amp, amp, size=pos.shape) / box


def mb_velocities(typ, masses, T, rng):
    m = np.asarray(masses, np.float64)[typ - 1]
    v = rng.standard_normal((len(typ), 3)) * np.sqrt(KB * T / m)[:, None]
    return v - v.mean(axis=0)


def ke_target(T):
    """Isokinetic target KE/N = 3/2 kB T (src/read_input.f90:230-231)."""
    return 1.5 * KB * T


def cu_crystal(n_cells=10, T=300.0, seed=1, quirk="ref"):
    """C1: FCC Cu, Morse, NVE."""
    rng = np.random.default_rng(seed)
    pos, box = lattice((n_cells,) * 3, CU_MORSE["a"], FCC_BASIS)
    typ = np.ones(len(pos), np.int32)
    vel = mb_velocities(typ, CU_MORSE["masses"], T, rng)
    return dict(name=f"cu_morse_fcc{n_cells}", masses=CU_MORSE["masses"],
                pairs=CU_MORSE["pairs"], typ=typ, pos=pos, box=box, vel=vel,
                control=dict(dt=0.1, skin=CU_MORSE["skin"], out_steps=100, quirk=quirk))


# A random FCC alloy with a one-sided pair: type 1 pushes type 2 through an
# 'asym' LJ line (PairMat(1,2) set, PairMat(2,1) not), so dynamics takes
# compute1 (src/nd.f90:155-163, 364-530); the like pairs are symmetric Morse.
ONESIDED = dict(masses=[63.546, 58.69],
                pairs=[(1, 1, True, "morse", [6.0, 0.3429, 1.3588, 2.866]),
                       (2, 2, True, "morse", [6.0, 0.4205, 1.4199, 2.780]),
                       (1, 2, False, "LJ", [6.0, 0.02, 2.4])],
                a=3.615, skin=0.5)


def onesided_alloy(n_cells=8, T=300.0, seed=7, quirk="fixed", frac2=0.4):
    """Random two-type FCC alloy with one one-sided (asym) pair, NVE."""
    rng = np.random.default_rng(seed)
    pos, box = lattice((n_cells,) * 3, ONESIDED["a"], FCC_BASIS)
    typ = np.where(rng.random(len(pos)) < frac2, 2, 1).astype(np.int32)
    vel = mb_velocities(typ, ONESIDED["masses"], T, rng)
    return dict(name=f"onesided_alloy{n_cells}", masses=ONESIDED["masses"],
                pairs=ONESIDED["pairs"], typ=typ, pos=pos, box=box, vel=vel,
                control=dict(dt=0.1, skin=ONESIDED["skin"], out_steps=100, quirk=quirk))


def spring_alloy(n_cells=8, T=300.0, seed=11, quirk="fixed", frac2=0.3, onesided=False):
    """Two-type FCC alloy whose type-1 nearest neighbours are bonded by
    strain springs ('spring' rc=3.0 A D0=4 eV/A sc=0.08 Vol=1, acting against
    the initial configuration: compute2, or compute3 when the type-1/type-2
    LJ line is one-sided); type-2 pairs are Morse."""
    rng = np.random.default_rng(seed)
    pos, box = lattice((n_cells,) * 3, ONESIDED["a"], FCC_BASIS)
    typ = np.where(rng.random(len(pos)) < frac2, 2, 1).astype(np.int32)
    vel = mb_velocities(typ, ONESIDED["masses"], T, rng)
    pairs = [(1, 1, True, "spring", [3.0, 4.0, 0.08, 1.0]),
             (2, 2, True, "morse", [6.0, 0.4205, 1.4199, 2.780]),
             (1, 2, not onesided, "LJ", [6.0, 0.02, 2.4])]
    return dict(name=f"spring_alloy{n_cells}", masses=ONESIDED["masses"], pairs=pairs,
                typ=typ, pos=pos, box=box, vel=vel,
                control=dict(dt=0.1, skin=0.5, out_steps=100, quirk=quirk))


def ar_liquid(n_cells=40, T=120.0, seed=2, quirk="fixed", thermostat=True):
    """C2: LJ argon at reduced density 0.8442, +-0.05 sigma jitter, NVT."""
    rng = np.random.default_rng(seed)
    pos, box = lattice((n_cells,) * 3, AR_LJ["a"], FCC_BASIS)
    pos = jitter(pos, box, 0.05 * 3.405, rng)
    typ = np.ones(len(pos), np.int32)
    vel = mb_velocities(typ, AR_LJ["masses"], T, rng)
    ctl = dict(dt=0.1, skin=AR_LJ["skin"], out_steps=100, quirk=quirk)
    if thermostat:
        ctl.update(isokinetic=1, ke_target=ke_target(T), ke_parm=100 * 0.1, ke_freq=1)
    return dict(name=f"ar_lj_fcc{n_cells}", masses=AR_LJ["masses"], pairs=AR_LJ["pairs"],
                typ=typ, pos=pos, box=box, vel=vel, control=ctl)


def nacl_solid(cells=(64, 64, 32), T=600.0, seed=3, quirk="fixed", p_parm=10.0):
    """C3: rocksalt two-species Buckingham solid, NPT (barostat + thermostat)."""
    rng = np.random.default_rng(seed)
    na, box = lattice(cells, NACL_BUCK["a"], ROCKSALT_NA)
    cl, _ = lattice(cells, NACL_BUCK["a"], ROCKSALT_CL)
    cl = (cl + 0.5) % 1.0 - 0.5
    pos = np.concatenate([na, cl])
    typ = np.concatenate([np.ones(len(na), np.int32), np.full(len(cl), 2, np.int32)])
    pos = jitter(pos, box, 0.02, rng)
    vel = mb_velocities(typ, NACL_BUCK["masses"], T, rng)
    ctl = dict(dt=0.1, skin=NACL_BUCK["skin"], out_steps=100, quirk=quirk,
               isokinetic=1, ke_target=ke_target(T), ke_parm=100 * 0.1, ke_freq=1,
               isobaric=1, p_target=[0.0, 0.0, 0.0], p_parm=p_parm, p_freq=1)
    return dict(name="nacl_buck_" + "x".join(map(str, cells)), masses=NACL_BUCK["masses"],
                pairs=NACL_BUCK["pairs"], typ=typ, pos=pos, box=box, vel=vel, control=ctl)


def replica_ensemble(nsys=512, seed=4, nmin=500, nmax=20000, quirk="fixed"):
    """C4: half Cu-Morse crystals, half LJ-Ar liquids; N log-uniform, FCC
    supercells rounded to whole cells (N = 4 n^3); T uniform in
    [100,1500] K, each with its own Berendsen thermostat."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(nsys):
        N = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        n = max(int(round((N / 4.0) ** (1.0 / 3.0))), 2)
        T = float(rng.uniform(100.0, 1500.0))
        sub = int(rng.integers(1 << 30))
        if s % 2 == 0:
            spec = cu_crystal(n, T, seed=sub, quirk=quirk)
        else:
            spec = ar_liquid(n, T, seed=sub, quirk=quirk)
        spec["control"].update(isokinetic=1, ke_target=ke_target(T), ke_parm=10.0, ke_freq=1)
        spec["T"] = T
        out.append(spec)
    return out


def serving_requests(nreq=4096, rate=200.0, seed=5, nmin=1000, nmax=200000, smin=1000,
                     smax=50000, quirk="fixed"):
    """C5 request stream: Poisson arrivals; potential, size, steps,
    temperature and ensemble drawn per request.  Returns light-weight
    descriptors; build_request() makes the system."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for r in range(nreq):
        t += rng.exponential(1.0 / rate)
        reqs.append(dict(id=r, arrival=t, pot=["morse", "lj", "buck"][int(rng.integers(3))],
                         natoms=math.exp(rng.uniform(math.log(nmin), math.log(nmax))),
                         steps=int(round(math.exp(rng.uniform(math.log(smin), math.log(smax))))),
                         T=float(rng.uniform(100.0, 1500.0)),
                         ensemble=["NVE", "NVT", "NPT"][int(rng.integers(3))],
                         seed=int(rng.integers(1 << 30)), quirk=quirk))
    return reqs


def build_request(r):
    N = r["natoms"]
    if r["pot"] == "buck":
        n = max(int(round((N / 8.0) ** (1.0 / 3.0))), 3)
        spec = nacl_solid((n, n, n), r["T"], r["seed"], quirk=r["quirk"])
        spec["control"].update(isobaric=0, isokinetic=0)
    elif r["pot"] == "lj":
        n = max(int(round((N / 4.0) ** (1.0 / 3.0))), 3)
        spec = ar_liquid(n, r["T"], r["seed"], quirk=r["quirk"], thermostat=False)
    else:
        n = max(int(round((N / 4.0) ** (1.0 / 3.0))), 3)
        spec = cu_crystal(n, r["T"], r["seed"], quirk=r["quirk"])
    ctl = spec["control"]
    if r["ensemble"] in ("NVT", "NPT"):
        ctl.update(isokinetic=1, ke_target=ke_target(r["T"]), ke_parm=10.0, ke_freq=1)
    if r["ensemble"] == "NPT":
        ctl.update(isobaric=1, p_target=[0.0, 0.0, 0.0], p_parm=10.0, p_freq=1)
    spec["steps"] = r["steps"]
    return spec


def add_to_context(ctx, spec, precision_tables=None):
    """Add a workload dict to a Context and apply its controls."""
    sid = ctx.add_system(spec["masses"], spec["pairs"], spec["typ"], spec["pos"], spec["box"],
                         vel=spec.get("vel"))
    ctx.set_control(sid, **spec["control"])
    return sid


def submit_to_server(srv, spec, nsteps=None):
    """Queue a workload dict on a Server; returns its ticket."""
    return srv.submit(spec["masses"], spec["pairs"], spec["typ"], spec["pos"], spec["box"],
                      int(nsteps if nsteps is not None else spec["steps"]), vel=spec.get("vel"),
                      **spec["control"])
