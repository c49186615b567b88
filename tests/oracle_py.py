"""ctypes binding of the CPU oracle (oracle/_build/libndyn_oracle.so).

Test infrastructure: used by tests/ as the parity checker and by bench.py's
cpu_baseline leg.  Never imported by the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ODIR = os.path.join(ROOT, "oracle")
LIB = os.path.join(ODIR, "_build", "libndyn_oracle.so")
# the same restatement built with the reference's release flags (-Ofast
# etc.): the timed CPU baseline only, never the parity checker
LIB_FAST = os.path.join(ODIR, "_build", "libndyn_oracle_fast.so")
EXE = os.path.join(ODIR, "_build", "ndyn_oracle")

MODE_REF, MODE_FIXED = 0, 1


def ensure_built():
    srcs = [os.path.join(ODIR, f) for f in ("ndyn_oracle.c", "ndyn_oracle.h", "ora_main.c")]
    if not (os.path.exists(LIB) and os.path.exists(EXE) and os.path.exists(LIB_FAST)) or any(
            os.path.getmtime(s) > os.path.getmtime(LIB) for s in srcs if os.path.exists(s)):
        subprocess.run(["make", "-s", "-C", ODIR], check=True)


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
                ("box_load", ctypes.c_int), ("box_vel", ctypes.c_double * 3)]


class Thermo(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int), ("potential", ctypes.c_double),
                ("kinetic", ctypes.c_double), ("energy_error", ctypes.c_double),
                ("pressure", ctypes.c_double), ("volume", ctypes.c_double),
                ("virial", ctypes.c_double * 6), ("box", ctypes.c_double * 3)]


THERMO_CB = ctypes.CFUNCTYPE(None, ctypes.POINTER(Thermo), ctypes.c_void_p)
_libs = {}


def lib(fast=False):
    """The parity build, or with fast=True the reference-flags build."""
    if fast not in _libs:
        ensure_built()
        L = ctypes.CDLL(LIB_FAST if fast else LIB)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.ora_new.restype = vp
        L.ora_free.argtypes = [vp]
        L.ora_set_threads.argtypes = [vp, i]
        L.ora_set_mode.argtypes = [vp, i]
        L.ora_set_types.argtypes = [vp, i, vp]
        L.ora_set_pairs.argtypes = [vp, i, d, i, vp, vp, vp, ctypes.c_char_p, vp, vp, vp]
        L.ora_get_tables.argtypes = [vp, vp, vp, vp, vp]
        L.ora_pot.argtypes = [ctypes.c_char_p, d, vp, d, d]
        L.ora_pot.restype = d
        L.ora_dpot.argtypes = [ctypes.c_char_p, d, vp, d, d]
        L.ora_dpot.restype = d
        L.ora_get_pairmat.argtypes = [vp, vp]
        L.ora_get_rcut.argtypes = [vp]
        L.ora_get_rcut.restype = d
        L.ora_set_state.argtypes = [vp, i, vp, vp, vp, vp, vp]
        L.ora_get_state.argtypes = [vp, vp, vp, vp, vp]
        L.ora_get_forces.argtypes = [vp, vp, vp, vp, vp]
        L.ora_default_control.argtypes = [ctypes.POINTER(Control)]
        L.ora_set_control.argtypes = [vp, ctypes.POINTER(Control)]
        L.ora_get_control.argtypes = [vp, ctypes.POINTER(Control)]
        for f in ("ora_setup_lists", "ora_build_cell_list", "ora_check_list_update",
                  "ora_get_list_updates", "ora_get_neimax"):
            getattr(L, f).argtypes = [vp]
        for f in ("ora_integrate1", "ora_mk_iso_ke", "ora_mk_iso_e", "ora_mk_iso_p"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = None
        L.ora_set_holds.argtypes = [vp, vp, i, vp, vp]
        L.ora_init_positions.argtypes = [vp, vp, vp]
        for f in ("ora_compute2", "ora_compute3"):
            getattr(L, f).argtypes = [vp, i, i]
            getattr(L, f).restype = None
        for f in ("ora_compute0", "ora_compute1", "ora_compute"):
            getattr(L, f).argtypes = [vp, i, i]
            getattr(L, f).restype = None
        L.ora_integrate2.argtypes = [vp, i]
        L.ora_integrate2.restype = None
        L.ora_run.argtypes = [vp, i, d, THERMO_CB, vp]
        L.ora_run_loop.argtypes = [vp, i, d, THERMO_CB, vp]
        L.ora_get_mcell.argtypes = [vp, vp]
        L.ora_get_cells.argtypes = [vp, vp]
        L.ora_get_neighbors.argtypes = [vp, vp, ctypes.c_long]
        L.ora_get_neighbors.restype = ctypes.c_long
        L.ora_get_skin.argtypes = [vp]
        L.ora_get_skin.restype = d
        L.ora_velocity.argtypes = [vp, ctypes.c_float, ctypes.c_ulonglong]
        L.ora_velocity.restype = None
        L.ora_fmt_thermo.argtypes = [ctypes.POINTER(Thermo), ctypes.c_char_p]
        L.ora_fmt_thermo.restype = None
        _libs[fast] = L
    return _libs[fast]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def pot(name, r, params, qprd=0.0, rcut=None):
    par = np.zeros(4)
    par[:len(params)] = params
    return lib().ora_pot(name.encode(), float(r), _p(par), float(qprd),
                         float(params[0] if rcut is None else rcut))


def dpot(name, r, params, qprd=0.0, rcut=None):
    par = np.zeros(4)
    par[:len(params)] = params
    return lib().ora_dpot(name.encode(), float(r), _p(par), float(qprd),
                          float(params[0] if rcut is None else rcut))


class Oracle:
    """One reference-semantics system (module globals of src/mods.f90)."""

    def __init__(self, threads=None, mode=MODE_REF, fast=False):
        self.L = lib(fast)
        self.s = ctypes.c_void_p(self.L.ora_new())
        if threads:
            self.L.ora_set_threads(self.s, int(threads))
        self.L.ora_set_mode(self.s, int(mode))
        self.np = 0
        self.ntypes = 0
        self.npairs = 0

    def __del__(self):
        try:
            self.L.ora_free(self.s)
        except Exception:
            pass

    def set_types(self, masses):
        m = np.ascontiguousarray(masses, dtype=np.float64)
        self.ntypes = len(m)
        assert self.L.ora_set_types(self.s, len(m), _p(m)) == 0

    def set_pairs(self, pairs, ptrmin=0.25, ptsize=1000, charges=None):
        """pairs: list of (t1, t2, sym, name, [params]) with 1-based types."""
        n = len(pairs)
        p1 = np.array([p[0] for p in pairs], np.int32)
        p2 = np.array([p[1] for p in pairs], np.int32)
        sym = np.array([1 if p[2] else 0 for p in pairs], np.int32)
        names = b"".join(p[3].encode().ljust(8)[:8] for p in pairs)
        par = np.zeros((n, 4))
        npar = np.zeros(n, np.int32)
        for k, p in enumerate(pairs):
            par[k, :len(p[4])] = p[4]
            npar[k] = len(p[4])
        q = np.zeros(n)
        if charges is not None:
            q = np.array([charges[p[0] - 1] * charges[p[1] - 1] for p in pairs])
        rc = self.L.ora_set_pairs(self.s, n, float(ptrmin), int(ptsize), _p(p1), _p(p2),
                                  _p(sym), names, _p(par), _p(npar), _p(q))
        assert rc == 0, rc
        self.npairs, self.ptsize = n, ptsize

    def tables(self):
        ts = (self.ptsize + 1) * self.npairs
        pp, fp = np.zeros(ts), np.zeros(ts)
        rc2, dr2 = np.zeros(self.npairs), np.zeros(self.npairs)
        self.L.ora_get_tables(self.s, _p(pp), _p(fp), _p(rc2), _p(dr2))
        return pp, fp, rc2, dr2

    def pairmat(self):
        pm = np.zeros(self.ntypes * self.ntypes, np.int32)
        self.L.ora_get_pairmat(self.s, _p(pm))
        return pm

    @property
    def rcut(self):
        return self.L.ora_get_rcut(self.s)

    def set_state(self, typ, pos, box, vel=None, acc=None):
        typ = np.ascontiguousarray(typ, np.int32)
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        box = np.ascontiguousarray(box, np.float64)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float64).reshape(-1)
        acc = None if acc is None else np.ascontiguousarray(acc, np.float64).reshape(-1)
        self.np = len(typ)
        assert self.L.ora_set_state(self.s, self.np, _p(typ), _p(pos), _p(vel), _p(acc),
                                    _p(box)) == 0

    def control(self):
        c = Control()
        self.L.ora_get_control(self.s, ctypes.byref(c))
        return c

    def set_control(self, **kw):
        c = self.control()
        for k, v in kw.items():
            if k in ("p_target", "box_vel"):
                for q in range(3):
                    getattr(c, k)[q] = v[q]
            else:
                setattr(c, k, v)
        assert self.L.ora_set_control(self.s, ctypes.byref(c)) == 0

    def velocity(self, kt, seed):
        self.L.ora_velocity(self.s, float(kt), int(seed))

    def state(self):
        n = self.np
        pos, vel, acc, box = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n), np.zeros(3)
        self.L.ora_get_state(self.s, _p(pos), _p(vel), _p(acc), _p(box))
        return pos.reshape(n, 3), vel.reshape(n, 3), acc.reshape(n, 3), box

    def forces(self):
        f = np.zeros(3 * self.np)
        pe, ke = ctypes.c_double(), ctypes.c_double()
        vir = np.zeros(6)
        self.L.ora_get_forces(self.s, _p(f), ctypes.byref(pe), _p(vir), ctypes.byref(ke))
        return f.reshape(self.np, 3), pe.value, vir, ke.value

    def setup_lists(self):
        return self.L.ora_setup_lists(self.s)

    def compute0(self, cv=1, cu=1):
        self.L.ora_compute0(self.s, cv, cu)

    def set_holds(self, hold, dirs, du):
        hold = np.ascontiguousarray(hold, np.int32)
        dirs = np.ascontiguousarray(np.asarray(dirs, bool).reshape(-1, 3), np.int32)
        du = np.ascontiguousarray(np.asarray(du, np.float64).reshape(-1, 3))
        assert self.L.ora_set_holds(self.s, _p(hold), len(du), _p(dirs), _p(du)) == 0

    def init_positions(self, ipos=None, ibox=None):
        ipos = None if ipos is None else np.ascontiguousarray(ipos, np.float64).reshape(-1)
        ibox = None if ibox is None else np.ascontiguousarray(ibox, np.float64)
        assert self.L.ora_init_positions(self.s, _p(ipos), _p(ibox)) == 0

    def compute(self, cv=1, cu=1):
        """The force routine dynamics would call: compute1 when some pair
        is one-sided, else compute0 (src/nd.f90:155-163)."""
        self.L.ora_compute(self.s, cv, cu)

    def integrate1(self):
        self.L.ora_integrate1(self.s)

    def integrate2(self, ck=1):
        self.L.ora_integrate2(self.s, ck)

    def check_list_update(self):
        return self.L.ora_check_list_update(self.s)

    def run(self, nsteps, dt, loop_only=False):
        """dynamics; loop_only skips the prologue (call setup_lists first)"""
        rows = []

        def cb(t, u):
            t = t.contents
            rows.append(dict(step=t.step, pe=t.potential, ke=t.kinetic,
                             eerr=t.energy_error, press=t.pressure, vol=t.volume,
                             virial=list(t.virial), box=list(t.box)))
        c = THERMO_CB(cb)
        fn = self.L.ora_run_loop if loop_only else self.L.ora_run
        rc = fn(self.s, int(nsteps), float(dt), c, None)
        return rc, rows

    def mcell(self):
        m = np.zeros(3, np.int32)
        self.L.ora_get_mcell(self.s, _p(m))
        return m

    def cells(self):
        c = np.zeros(self.np, np.int32)
        assert self.L.ora_get_cells(self.s, _p(c)) == 0
        return c

    def neighbors(self):
        n = self.L.ora_get_neighbors(self.s, None, 0)
        pairs = np.zeros(2 * max(n, 1), np.int32)
        self.L.ora_get_neighbors(self.s, _p(pairs), n)
        return pairs[:2 * n].reshape(n, 2)

    @property
    def list_updates(self):
        return self.L.ora_get_list_updates(self.s)

    @property
    def skin(self):
        return self.L.ora_get_skin(self.s)

    @property
    def neimax(self):
        return self.L.ora_get_neimax(self.s)


def fmt_thermo(row):
    t = Thermo()
    t.step = row["step"]
    t.potential, t.kinetic = row["pe"], row["ke"]
    t.energy_error, t.pressure, t.volume = row["eerr"], row["press"], row["vol"]
    buf = ctypes.create_string_buffer(96)
    lib().ora_fmt_thermo(ctypes.byref(t), buf)
    return buf.value.decode()


def run_script(script_lines, cwd, fixed=False, threads=None):
    """Run a directive script through the oracle driver; return thermo rows."""
    ensure_built()
    args = [EXE] + (["--fixed"] if fixed else []) + (
        ["--threads", str(threads)] if threads else [])
    r = subprocess.run(args, input="START\n" + "\n".join(script_lines) + "\n",
                       text=True, capture_output=True, cwd=cwd)
    rows = []
    for ln in r.stdout.splitlines():
        w = ln.split()
        if len(w) == 6 and w[0].isdigit():
            rows.append(dict(step=int(w[0]), pe=float(w[1]), ke=float(w[2]),
                             eerr=float(w[3]), press=float(w[4]), vol=float(w[5]), text=ln))
    return r.returncode, rows, r.stdout, r.stderr
