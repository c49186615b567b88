"""Python mirror of the Ndyn timestep interface over the C ABI (ndyn_gpu.h).

The reference's timestep routines are Fortran subroutines on module state
(stewmasterj/Ndyn_OMP src/nd.f90).  `Context` holds that state on the GPU
for one or more independent systems and exposes one method per routine,
with the reference's names and flag arguments:

    ctx.setup_lists()          dynamics prologue     src/nd.f90:73-108
    ctx.build_cell_list()      buildCellList         src/nd.f90:1214-1260
    ctx.check_list_update()    CheckListUpdate       src/nd.f90:1447-1499
    ctx.integrate1()           integrate1            src/nd.f90:984-1080
    ctx.compute0(cv, cu)       compute0(CV,CU)       src/nd.f90:200-363
    ctx.integrate2(ck)         integrate2(CK)        src/nd.f90:1081-1121
    ctx.mk_iso_ke/e/p(sys)     mkIsoKE/mkIsoE/mkIsoP src/nd.f90:1122-1213
    ctx.run(nsteps)            the dynamics loop     src/nd.f90:137-180

`Server` is the serving loop (continuous batching of independent runs, no
counterpart in the reference): submit(), step(), poll(), result().

Errors the reference reports with STOP raise NdgError with the library's
status code.  Everything runs in the CUDA library; there is no CPU path.
"""
import ctypes
import os

import numpy as np

from . import _lib as L

PREC = {"fp64": 0, "mixed": 1}
QUIRK = {"ref": 0, "fixed": 1}


class NdgError(RuntimeError):
    def __init__(self, status, what=""):
        lib = L.lib()
        msg = lib.ndg_error_string(status).decode()
        detail = lib.ndg_last_error(None).decode() if status == -7 else ""
        super().__init__(f"{what}: {msg} ({status}) {detail}".strip())
        self.status = status


def _ok(status, what=""):
    if status != 0:
        raise NdgError(status, what)


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def build_pair_tables(pairs, ptsize=1000, ptrmin=0.25, charges=None):
    """buildPairTables (src/potentials.f90:2-56) for a list of pair specs.

    pairs: sequence of (type_i, type_j, sym, name, params) with 1-based
    types and params = [rc, p2, p3, p4] as on a 'Pairs' line.  Returns
    (ppair, fpair, rc2, dr2) with the reference's (PTsize+1, NPairs)
    column-major tables flattened."""
    n = len(pairs)
    names = b"".join(p[3].encode().ljust(8)[:8] for p in pairs)
    par = np.zeros((n, 4))
    for k, p in enumerate(pairs):
        par[k, :len(p[4])] = p[4]
    q = None
    if charges is not None:
        q = np.array([charges[p[0] - 1] * charges[p[1] - 1] for p in pairs], np.float64)
    pp = np.zeros((ptsize + 1) * n)
    fp = np.zeros((ptsize + 1) * n)
    rc2 = np.zeros(n)
    dr2 = np.zeros(n)
    _ok(L.lib().ndg_build_pair_tables(n, ptsize, float(ptrmin), names, _p(par), _p(q), _p(pp),
                                      _p(fp), _p(rc2), _p(dr2)), "build_pair_tables")
    return pp, fp, rc2, dr2


def pair_matrix(pairs, ntypes):
    """PairMat(ntypes,ntypes), column-major, as the 'Pairs' directive fills
    it (src/read_input.f90:159-164)."""
    pm = np.zeros((ntypes, ntypes), np.int32)  # pm[a-1, b-1] = PairMat(a,b)
    for k, p in enumerate(pairs):
        pm[p[0] - 1, p[1] - 1] = k + 1
        if p[2]:
            pm[p[1] - 1, p[0] - 1] = k + 1
    return np.asfortranarray(pm).ravel(order="F")


class Control(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("skin", ctypes.c_double),
                ("neimax", ctypes.c_int), ("renei", ctypes.c_int),
                ("renei_freq", ctypes.c_int), ("out_steps", ctypes.c_int),
                ("step", ctypes.c_int),
                ("isokinetic", ctypes.c_int), ("ke_freq", ctypes.c_int),
                ("ke_target", ctypes.c_double), ("ke_parm", ctypes.c_double),
                ("isobaric", ctypes.c_int), ("p_freq", ctypes.c_int),
                ("p_target", ctypes.c_double * 3), ("p_parm", ctypes.c_double),
                ("isoenergetic", ctypes.c_int), ("e_freq", ctypes.c_int),
                ("e_parm", ctypes.c_double),
                ("box_load", ctypes.c_int), ("box_vel", ctypes.c_double * 3),
                ("quirk", ctypes.c_int)]


class Thermo(ctypes.Structure):
    _fields_ = [("sys", ctypes.c_int), ("step", ctypes.c_int),
                ("potential", ctypes.c_double), ("kinetic", ctypes.c_double),
                ("energy_error", ctypes.c_double), ("pressure", ctypes.c_double),
                ("volume", ctypes.c_double), ("virial", ctypes.c_double * 6),
                ("box", ctypes.c_double * 3)]

    def as_dict(self):
        return dict(sys=self.sys, step=self.step, pe=self.potential, ke=self.kinetic,
                    eerr=self.energy_error, press=self.pressure, vol=self.volume,
                    virial=list(self.virial), box=list(self.box))


THERMO_CB = ctypes.CFUNCTYPE(None, ctypes.POINTER(Thermo), ctypes.c_void_p)


class Context:
    """A GPU context holding one or more independent systems."""

    def __init__(self, device=0, precision="fp64"):
        self.L = L.lib()
        self._c = ctypes.c_void_p()
        _ok(self.L.ndg_create(ctypes.byref(self._c), int(device), PREC[precision]), "create")
        self.systems = {}

    def close(self):
        if self._c:
            self.L.ndg_destroy(self._c)
            self._c = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- systems ---------------------------------------------------------
    def add_system(self, masses, pairs, typ, pos, box, vel=None, acc=None, ptsize=1000,
                   ptrmin=0.25, charges=None, tables=None):
        """Add one system; pairs as for build_pair_tables, pos (np,3)
        fractional.  tables=(ppair, fpair) supplies the caller's own tables."""
        masses = np.ascontiguousarray(masses, np.float64)
        nt = len(masses)
        if tables is None:
            pp, fp, _, _ = build_pair_tables(pairs, ptsize, ptrmin, charges)
        else:
            pp, fp = (np.ascontiguousarray(t, np.float64) for t in tables)
        pm = pair_matrix(pairs, nt)
        rcp = np.array([p[4][0] for p in pairs], np.float64)
        typ = np.ascontiguousarray(typ, np.int32)
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float64).reshape(-1)
        acc = None if acc is None else np.ascontiguousarray(acc, np.float64).reshape(-1)
        box = np.ascontiguousarray(box, np.float64)
        sid = ctypes.c_int()
        _ok(self.L.ndg_add_system(self._c, len(typ), nt, len(pairs), int(ptsize), float(ptrmin),
                                  _p(masses), _p(pm), _p(rcp), _p(pp), _p(fp), _p(typ), _p(pos),
                                  _p(vel), _p(acc), _p(box), ctypes.byref(sid)), "add_system")
        self.systems[sid.value] = len(typ)
        if any(p[3] == "spring" for p in pairs):
            # PairParams(1:4) of each spring line: rc, D0, sc, Vol
            flags = np.array([1 if p[3] == "spring" else 0 for p in pairs], np.int32)
            prm = np.zeros((len(pairs), 4))
            for k, p in enumerate(pairs):
                prm[k, :len(p[4])] = p[4][:4]
            _ok(self.L.ndg_set_springs(self._c, sid.value, _p(flags), _p(prm)), "set_springs")
        return sid.value

    def set_initial_positions(self, sys, ipos=None, ibox=None):
        """InitPos: the spring strains' initial positions (np,3) fractional
        and box; None takes the current ones."""
        ipos = None if ipos is None else np.ascontiguousarray(ipos, np.float64).reshape(-1)
        ibox = None if ibox is None else np.ascontiguousarray(ibox, np.float64)
        _ok(self.L.ndg_set_initial_positions(self._c, sys, _p(ipos), _p(ibox)),
            "set_initial_positions")

    def remove_system(self, sys):
        _ok(self.L.ndg_remove_system(self._c, sys), "remove_system")
        self.systems.pop(sys, None)

    def control(self, sys=0):
        c = Control()
        _ok(self.L.ndg_get_control(self._c, sys, ctypes.byref(c)), "get_control")
        return c

    def set_control(self, sys=0, **kw):
        c = self.control(sys)
        for k, v in kw.items():
            if k == "quirk" and isinstance(v, str):
                v = QUIRK[v]
            if k in ("p_target", "box_vel"):
                for q in range(3):
                    getattr(c, k)[q] = v[q]
            else:
                setattr(c, k, v)
        _ok(self.L.ndg_set_control(self._c, sys, ctypes.byref(c)), "set_control")

    def set_holds(self, sys, hold=None, dirs=None, du=None):
        """Hold groups with displacement conditions (Hold/Disp directives,
        integrate1's Nhold branch): hold[i] in 0..G per atom in input order,
        dirs (G,3) booleans, du (G,3) fractional displacement per step.
        hold=None removes them."""
        if hold is None:
            _ok(self.L.ndg_set_holds(self._c, sys, None, 0, None, None), "set_holds")
            return
        hold = np.ascontiguousarray(hold, np.int32)
        dirs = np.ascontiguousarray(np.asarray(dirs, bool).reshape(-1, 3), np.int32)
        du = np.ascontiguousarray(np.asarray(du, np.float64).reshape(-1, 3))
        _ok(self.L.ndg_set_holds(self._c, sys, _p(hold), len(du), _p(dirs), _p(du)), "set_holds")

    def load_state(self, sys, pos, vel=None, acc=None, box=None):
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float64).reshape(-1)
        acc = None if acc is None else np.ascontiguousarray(acc, np.float64).reshape(-1)
        box = None if box is None else np.ascontiguousarray(box, np.float64)
        _ok(self.L.ndg_load_state(self._c, sys, _p(pos), _p(vel), _p(acc), _p(box)), "load_state")

    def state(self, sys=0):
        n = self.systems[sys]
        pos, vel, acc, box = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n), np.zeros(3)
        _ok(self.L.ndg_get_state(self._c, sys, _p(pos), _p(vel), _p(acc), _p(box)), "get_state")
        return pos.reshape(n, 3), vel.reshape(n, 3), acc.reshape(n, 3), box

    def load_states(self, pos, vel=None, acc=None, boxes=None):
        """Every live system at once (ndg_load_state with sys = -1): pos,
        vel, acc are (sum of np, 3) arrays holding the systems one after
        another in ascending id order, boxes (nsys, 3).  Page-locked arrays
        (e.g. from torch's pin_memory) move by DMA."""
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float64).reshape(-1)
        acc = None if acc is None else np.ascontiguousarray(acc, np.float64).reshape(-1)
        boxes = None if boxes is None else np.ascontiguousarray(boxes, np.float64).reshape(-1)
        _ok(self.L.ndg_load_state(self._c, -1, _p(pos), _p(vel), _p(acc), _p(boxes)),
            "load_state(all)")

    def states(self, out=None):
        """Every live system's (pos, vel, acc) as (sum of np, 3) arrays in
        ascending id order, and boxes (nsys, 3) (ndg_get_state with sys = -1).
        out = (pos, vel, acc, boxes) writes into the caller's arrays."""
        total = sum(self.systems.values())
        if out is None:
            out = (np.zeros((total, 3)), np.zeros((total, 3)), np.zeros((total, 3)),
                   np.zeros((len(self.systems), 3)))
        pos, vel, acc, boxes = out
        _ok(self.L.ndg_get_state(self._c, -1, _p(pos), _p(vel), _p(acc), _p(boxes)),
            "get_state(all)")
        return pos, vel, acc, boxes

    def forces(self, sys=0):
        n = self.systems[sys]
        f = np.zeros(3 * n)
        pe, ke = ctypes.c_double(), ctypes.c_double()
        vir = np.zeros(6)
        _ok(self.L.ndg_get_forces(self._c, sys, _p(f), ctypes.byref(pe), _p(vir),
                                  ctypes.byref(ke)), "get_forces")
        return f.reshape(n, 3), pe.value, vir, ke.value

    # -- the reference routines ---------------------------------------------
    def setup_lists(self):
        _ok(self.L.ndg_setup_lists(self._c), "setup_lists")

    def build_cell_list(self):
        _ok(self.L.ndg_build_cell_list(self._c), "build_cell_list")

    def check_list_update(self):
        n = ctypes.c_int()
        _ok(self.L.ndg_check_list_update(self._c, ctypes.byref(n)), "check_list_update")
        return n.value

    def integrate1(self):
        _ok(self.L.ndg_integrate1(self._c), "integrate1")

    def compute0(self, cv=True, cu=True):
        _ok(self.L.ndg_compute(self._c, int(cv), int(cu)), "compute0")

    def integrate2(self, ck=True):
        _ok(self.L.ndg_integrate2(self._c, int(ck)), "integrate2")

    def mk_iso_ke(self, sys=0):
        _ok(self.L.ndg_mk_iso_ke(self._c, sys), "mkIsoKE")

    def mk_iso_e(self, sys=0):
        _ok(self.L.ndg_mk_iso_e(self._c, sys), "mkIsoE")

    def mk_iso_p(self, sys=0):
        _ok(self.L.ndg_mk_iso_p(self._c, sys), "mkIsoP")

    def run(self, nsteps, callback=None, cont=False):
        """The dynamics loop; returns every write_thermo record as a dict."""
        rows = []

        def cb(t, u):
            d = t.contents.as_dict()
            rows.append(d)
            if callback:
                callback(d)
        c = THERMO_CB(cb)
        fn = self.L.ndg_run_continue if cont else self.L.ndg_run
        _ok(fn(self._c, int(nsteps), c, None), "run")
        return rows

    def thermo(self, sys=0):
        t = Thermo()
        _ok(self.L.ndg_get_thermo(self._c, sys, ctypes.byref(t)), "get_thermo")
        return t.as_dict()

    def list_updates(self, sys=0):
        n = ctypes.c_int()
        _ok(self.L.ndg_get_list_updates(self._c, sys, ctypes.byref(n)), "list_updates")
        return n.value

    # -- inspection -----------------------------------------------------------
    def mcell(self, sys=0):
        m = np.zeros(3, np.int32)
        _ok(self.L.ndg_get_mcell(self._c, sys, _p(m)), "get_mcell")
        return m

    def cells(self, sys=0):
        c = np.zeros(self.systems[sys], np.int32)
        _ok(self.L.ndg_get_cells(self._c, sys, _p(c)), "get_cells")
        return c

    def neighbor_count(self, sys=0):
        """entries of the full neighbour list (each pair from both atoms)"""
        n = ctypes.c_longlong()
        _ok(self.L.ndg_get_neighbor_count(self._c, sys, ctypes.byref(n)), "get_neighbor_count")
        return n.value

    def neighbors(self, sys=0):
        n = ctypes.c_longlong()
        _ok(self.L.ndg_get_neighbors(self._c, sys, None, 0, ctypes.byref(n)), "get_neighbors")
        pairs = np.zeros(2 * max(n.value, 1), np.int32)
        _ok(self.L.ndg_get_neighbors(self._c, sys, _p(pairs), n.value, ctypes.byref(n)),
            "get_neighbors")
        return pairs[:2 * n.value].reshape(-1, 2)

    # -- timing -----------------------------------------------------------------
    @property
    def stream_ptr(self):
        """cudaStream_t of the library's launches (for CUDA events)"""
        p = ctypes.c_void_p()
        _ok(self.L.ndg_get_stream(self._c, ctypes.byref(p)), "get_stream")
        return p.value

    def profile_run(self, nsteps):
        """continue the run eagerly with events around each kernel group;
        returns mean ms per launch (integrate1, pair, rebuild group)"""
        _ok(self.L.ndg_profile_run(self._c, int(nsteps)), "profile_run")
        ti, tp, tr = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        n = ctypes.c_int()
        _ok(self.L.ndg_get_kernel_times(self._c, ctypes.byref(ti), ctypes.byref(tp),
                                        ctypes.byref(tr), ctypes.byref(n)), "kernel_times")
        return dict(integrate_ms=ti.value, pair_ms=tp.value, rebuild_ms=tr.value,
                    launches=n.value)

    # -- tuning ---------------------------------------------------------------
    def set_tuning(self, tpa=0, graph_steps=100):
        _ok(self.L.ndg_set_tuning(self._c, int(tpa), int(graph_steps)), "set_tuning")

    def tuning(self):
        t, g = ctypes.c_int(), ctypes.c_int()
        _ok(self.L.ndg_get_tuning(self._c, ctypes.byref(t), ctypes.byref(g)), "get_tuning")
        return t.value, g.value

    def set_gather_depth(self, depth):
        _ok(self.L.ndg_set_gather_depth(self._c, int(depth)), "set_gather_depth")

    def gather_depth(self):
        d = ctypes.c_int()
        _ok(self.L.ndg_get_gather_depth(self._c, ctypes.byref(d)), "get_gather_depth")
        return d.value

    def autotune(self, steps=20):
        _ok(self.L.ndg_autotune(self._c, int(steps)), "autotune")
        return self.tuning()

    def set_list_split(self, rows, tpa_long=2):
        """atoms to threads by list length (ndg_set_list_split): systems whose
        mean list length reaches `rows` run with `tpa_long` threads per atom;
        rows = 0: one class"""
        _ok(self.L.ndg_set_list_split(self._c, int(rows), int(tpa_long)), "set_list_split")

    def list_split(self):
        """(rows threshold, threads per atom of the long-list class)"""
        r, t = ctypes.c_int(), ctypes.c_int()
        _ok(self.L.ndg_get_list_split(self._c, ctypes.byref(r), ctypes.byref(t)), "get_list_split")
        return r.value, t.value

    def autotune_skin(self, steps=60):
        """The rebuild-interval autotuner (ndg_autotune_skin): a list skin
        per fixed-semantics system from a trial of `steps` steps, which is
        undone; returns the number of systems whose skin changed."""
        n = ctypes.c_int()
        _ok(self.L.ndg_autotune_skin(self._c, int(steps), ctypes.byref(n)), "autotune_skin")
        return n.value

    def set_precision(self, precision):
        _ok(self.L.ndg_set_precision(self._c, PREC[precision]), "set_precision")


# ---------------------------------------------------------------------------
class Request(ctypes.Structure):
    _fields_ = [("np", ctypes.c_int), ("ntypes", ctypes.c_int), ("npairs", ctypes.c_int),
                ("ptsize", ctypes.c_int), ("ptrmin", ctypes.c_double),
                ("mass", ctypes.c_void_p), ("pairmat", ctypes.c_void_p),
                ("rcpair", ctypes.c_void_p), ("ppair", ctypes.c_void_p),
                ("fpair", ctypes.c_void_p), ("typ", ctypes.c_void_p), ("pos", ctypes.c_void_p),
                ("vel", ctypes.c_void_p), ("box", ctypes.c_void_p), ("control", Control),
                ("nsteps", ctypes.c_int), ("spring", ctypes.c_void_p),
                ("pair_params", ctypes.c_void_p)]


class ServerStats(ctypes.Structure):
    _fields_ = [("queued", ctypes.c_int), ("resident", ctypes.c_int),
                ("completed", ctypes.c_int), ("failed", ctypes.c_int),
                ("bytes_in_use", ctypes.c_longlong), ("budget", ctypes.c_longlong),
                ("atom_steps", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_setup", ctypes.c_double), ("t_block", ctypes.c_double),
                ("t_retire", ctypes.c_double), ("graph_captures", ctypes.c_int),
                ("blocks", ctypes.c_int)]


def make_control(**kw):
    """An ndg_control with the reference's defaults, then the given fields."""
    c = Control()
    L.lib().ndg_default_control(ctypes.byref(c))
    for k, v in kw.items():
        if k == "quirk" and isinstance(v, str):
            v = QUIRK[v]
        if k in ("p_target", "box_vel"):
            for q in range(3):
                getattr(c, k)[q] = v[q]
        else:
            setattr(c, k, v)
    return c


def admit_plan(nbytes, budget, in_use=0):
    """The server's admission rule on its own (host only): which queued
    requests, in order, fit what is left of the budget."""
    b = np.ascontiguousarray(nbytes, np.int64)
    out = np.zeros(len(b), np.int32)
    k = L.lib().ndg_admit_plan(_p(b), len(b), int(budget), int(in_use), _p(out))
    if k < 0:
        raise NdgError(k, "admit_plan")
    return out.astype(bool)


class Server:
    """Continuous batching of independent MD runs on one GPU.

    submit() queues a run (its arrays are copied); each step() admits queued
    runs that fit the HBM budget, builds their lists, and advances every
    resident run by one block of block_steps steps; finished runs are
    retired and their final state waits for result()."""

    def __init__(self, device=0, precision="mixed", hbm_budget=150e9, block_steps=100):
        self.L = L.lib()
        self._s = ctypes.c_void_p()
        _ok(self.L.ndg_server_create(ctypes.byref(self._s), int(device), PREC[precision],
                                     int(hbm_budget), int(block_steps)), "server_create")
        self.natoms = {}

    def close(self):
        if self._s:
            self.L.ndg_server_destroy(self._s)
            self._s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, masses, pairs, typ, pos, box, nsteps, vel=None, ptsize=1000, ptrmin=0.25,
               **control):
        masses = np.ascontiguousarray(masses, np.float64)
        nt = len(masses)
        pp, fp, _, _ = build_pair_tables(pairs, ptsize, ptrmin)
        pm = pair_matrix(pairs, nt)
        rcp = np.array([p[4][0] for p in pairs], np.float64)
        typ = np.ascontiguousarray(typ, np.int32)
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float64).reshape(-1)
        box = np.ascontiguousarray(box, np.float64)
        spring = prm = None
        if any(p[3] == "spring" for p in pairs):
            spring = np.array([1 if p[3] == "spring" else 0 for p in pairs], np.int32)
            prm = np.zeros((len(pairs), 4))
            for k, p in enumerate(pairs):
                prm[k, :len(p[4])] = p[4][:4]
        r = Request(np=len(typ), ntypes=nt, npairs=len(pairs), ptsize=int(ptsize),
                    ptrmin=float(ptrmin), mass=_p(masses), pairmat=_p(pm), rcpair=_p(rcp),
                    ppair=_p(pp), fpair=_p(fp), typ=_p(typ), pos=_p(pos), vel=_p(vel),
                    box=_p(box), control=make_control(**control), nsteps=int(nsteps),
                    spring=_p(spring), pair_params=_p(prm))
        t = ctypes.c_longlong()
        _ok(self.L.ndg_server_submit(self._s, ctypes.byref(r), ctypes.byref(t)), "server_submit")
        # write_thermo rows: every OutSteps-th step and the run's first
        self.natoms[t.value] = (len(typ), int(nsteps) // max(r.control.out_steps, 1) + 2)
        return t.value

    def step(self):
        """admit what fits, one block for every resident run; returns the
        number of runs that finished in this call"""
        n = ctypes.c_int()
        _ok(self.L.ndg_server_step(self._s, ctypes.byref(n)), "server_step")
        return n.value

    def poll(self):
        out = []
        buf = (ctypes.c_longlong * 256)()
        while True:
            n = ctypes.c_int()
            _ok(self.L.ndg_server_poll(self._s, buf, 256, ctypes.byref(n)), "server_poll")
            out.extend(buf[k] for k in range(n.value))
            if n.value < 256:
                return out

    def status(self, ticket):
        st = ctypes.c_int()
        _ok(self.L.ndg_server_status(self._s, int(ticket), ctypes.byref(st)), "server_status")
        return st.value

    def result(self, ticket):
        """(pos, vel, acc, box, thermo rows) of a finished run"""
        n, cap = self.natoms.pop(ticket)
        pos, vel, acc, box = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n), np.zeros(3)
        rows = (Thermo * cap)()
        nrows = ctypes.c_int()
        _ok(self.L.ndg_server_result(self._s, int(ticket), _p(pos), _p(vel), _p(acc), _p(box),
                                     rows, cap, ctypes.byref(nrows)), "server_result")
        out = [rows[k].as_dict() for k in range(min(cap, nrows.value))]
        return pos.reshape(n, 3), vel.reshape(n, 3), acc.reshape(n, 3), box, out

    def stats(self):
        st = ServerStats()
        _ok(self.L.ndg_server_stats_get(self._s, ctypes.byref(st)), "server_stats")
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    @property
    def stream_ptr(self):
        c = ctypes.c_void_p()
        _ok(self.L.ndg_server_context(self._s, ctypes.byref(c)), "server_context")
        p = ctypes.c_void_p()
        _ok(self.L.ndg_get_stream(c, ctypes.byref(p)), "get_stream")
        return p.value
