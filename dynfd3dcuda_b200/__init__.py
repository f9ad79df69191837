"""B200-native curved-grid finite-difference dynamic-rupture time step.

Python mirror of the C ABI in include/dfd_b200.h (libdfd_b200.so, built in-tree by
dynfd3dcuda_b200/build.py).  The job dictionary uses the reference's params.json keys
(set_params.cu:137-282); input arrays use the reference's file layouts:

    fxyz    (3, NZ, NY) float32   Fault_geometry x, y, z
    stress  (15, NZ, NY) float32  Fault_init_stress Tx Ty Tz dTx dTy dTz mu_s mu_d Dc C0 a b L Vw State
            (16, NZ, NY)          the same plus TP_hy, for Friction_type 3
    layers  (n, 4) float32        Media1D rows depth rho vp vs

There is no CPU fallback: constructing a Simulation without the CUDA library or without
a GPU raises.
"""
import ctypes
import json
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libdfd_b200.so")
_lib = None

FIELDS = ["slip", "hslip", "Vs1", "Vs2", "Tn", "Ts1", "Ts2", "State", "init_t0", "tTn", "tTs1", "tTs2",
          "str_peak", "friction", "united", "faultgrid", "split", "T1", "hT1", "TP_T", "TP_P", "rup_sensor"]
HALO_SETUP = 4  # dfd_halo_pack / dfd_halo_unpack: the metric and media of the ghost columns

# coefficient tables of dfd_get_fault_table, in the order of the DFD_TAB_* names
TABLES = ["D21_1", "D22_1", "D23_1", "D31_1", "D32_1", "D33_1", "D21_2", "D22_2", "D23_2", "D31_2", "D32_2", "D33_2",
          "matMin2Plus1", "matMin2Plus2", "matMin2Plus3", "matMin2Plus4", "matMin2Plus5",
          "matPlus2Min1", "matPlus2Min2", "matPlus2Min3", "matPlus2Min4", "matPlus2Min5",
          "matT1toVxm", "matVytoVxm", "matVztoVxm", "matT1toVxp", "matVytoVxp", "matVztoVxp",
          "matVx2Vz1", "matVy2Vz1", "matVx2Vz2", "matVy2Vz2", "matPlus2Min1f", "matPlus2Min2f", "matPlus2Min3f",
          "matMin2Plus1f", "matMin2Plus2f", "matMin2Plus3f", "vec_n", "vec_s1", "vec_s2"]
STATUS = {0: "ok", 1: "bad or unsupported parameter", 2: "CUDA error", 3: "file missing or malformed",
          4: "call out of order", 5: "DT above the stability limit", 6: "non-finite fault state",
          7: "Newton solve hit its iteration cap"}


class Ensemble:
    """Prepared Simulations on one device stepped together (dfd_ens_*): one batched launch
    per kernel and RK stage over all scenarios, replayed from CUDA graphs.  The scenarios
    keep their state; read it from the Simulation objects."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (ctypes.c_void_p * len(self.sims))(*[s.h.value if hasattr(s.h, "value") else s.h for s in self.sims])
        h = ctypes.c_void_p()
        r = lib().dfd_ens_create(arr, len(self.sims), ctypes.byref(h))
        if r:
            raise DfdError(r, "dfd_ens_create")
        self.h = h

    def _check(self, r):
        if r:
            lib().dfd_ens_last_error.restype = ctypes.c_char_p
            lib().dfd_ens_last_error.argtypes = [ctypes.c_void_p]
            raise DfdError(r, (lib().dfd_ens_last_error(self.h) or b"").decode())

    def run(self, it0, nsteps):
        self._check(lib().dfd_ens_run(self.h, it0, nsteps))

    def synchronize(self):
        self._check(lib().dfd_ens_synchronize(self.h))

    def run_timed(self, it0, nsteps):
        """Device time (ms) of nsteps steps."""
        ms = ctypes.c_float()
        self._check(lib().dfd_ens_run_timed(self.h, it0, nsteps, ctypes.byref(ms)))
        return ms.value

    def set_chunk(self, chunk):
        """x planes per unit of the tiled kernel (0: each scenario's own plan)."""
        self._check(lib().dfd_ens_set_chunk(self.h, int(chunk)))

    def set_tile_rows(self, rows):
        """Rows of the interior kernel's tiles for every scenario: 8 (one CTA per SM) or 4
        (two CTAs per SM)."""
        self._check(lib().dfd_ens_set_tile_rows(self.h, int(rows)))

    def nodes(self):
        n = ctypes.c_longlong()
        self._check(lib().dfd_ens_nodes(self.h, ctypes.byref(n)))
        return n.value

    def autotune(self, it0, candidates=(0, 16, 32, 64, 128), steps=4, rows=(8, 4)):
        """Time a few steps with each layout of the interior kernel's units, a tile shape
        (rows of a 32-wide tile, with the CTAs per SM it allows) times a unit length (x
        planes, 0: each scenario's own plan), and keep the fastest.  Returns
        ({(rows, chunk): ms}, best (rows, chunk), next step).  The steps are real steps: the
        scenarios advance by (1 + steps) per candidate."""
        times = {}
        it = it0
        for r in rows:
            self.set_tile_rows(r)
            for c in candidates:
                self.set_chunk(c)
                self.run(it, 1)  # graphs of this layout
                it += 1
                times[(r, c)] = self.run_timed(it, steps)
                it += steps
        best = min(times, key=times.get)
        self.set_tile_rows(best[0])
        self.set_chunk(best[1])
        return times, best, it

    def close(self):
        if getattr(self, "h", None):
            lib().dfd_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


# parameter vector of the learned Newton guess (DFD_MLP_PARAMS, DFD_MLP_TRAINABLE)
MLP_PARAMS = 1259
MLP_TRAINABLE = 1249


def _check(r):
    if r:
        raise DfdError(r)


def mlp_init(seed, x_mean, x_scale, y_mean, y_scale):
    """Initial parameter vector: Xavier weights from seed, standardisation constants."""
    w = np.zeros(MLP_PARAMS, np.float32)
    xm = np.ascontiguousarray(x_mean, np.float32)
    xs = np.ascontiguousarray(x_scale, np.float32)
    _check(lib().dfd_mlp_init(w.ctypes.data, int(seed), xm.ctypes.data, xs.ctypes.data, float(y_mean), float(y_scale)))
    return w


def mlp_forward(w, x):
    """Residual predicted by the network for inputs x (n, 4), on the GPU."""
    w = np.ascontiguousarray(w, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty(len(x), np.float32)
    _check(lib().dfd_mlp_forward(w.ctypes.data, x.ctypes.data, len(x), y.ctypes.data))
    return y


def mlp_forward_node(w, x, tensor_cores=True):
    """Residuals from the fault node kernel's own inference (per-thread or tensor-core
    network) for inputs x (n, 4), on the GPU."""
    w = np.ascontiguousarray(w, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty(len(x), np.float32)
    _check(lib().dfd_mlp_forward_node(w.ctypes.data, x.ctypes.data, len(x), int(tensor_cores), y.ctypes.data))
    return y


def mlp_loss_grad(w, x, y):
    """(mean squared standardised error, gradient over the MLP_TRAINABLE weights), on the GPU."""
    w = np.ascontiguousarray(w, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    g = np.empty(MLP_TRAINABLE, np.float32)
    loss = ctypes.c_double()
    _check(lib().dfd_mlp_loss_grad(w.ctypes.data, x.ctypes.data, y.ctypes.data, len(x), ctypes.byref(loss),
                                   g.ctypes.data))
    return loss.value, g


def mlp_train(w, x, y, epochs, batch=4096, lr=3e-3, seed=0):
    """Minibatch Adam on the GPU; returns (trained weights, loss per epoch)."""
    w = np.array(w, np.float32, copy=True)
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    hist = np.zeros(epochs, np.float32)
    _check(lib().dfd_mlp_train(x.ctypes.data, y.ctypes.data, len(x), int(epochs), int(batch), float(lr), int(seed),
                               w.ctypes.data, hist.ctypes.data))
    return w, hist


def train_guess_net(samples, epochs=8, batch=4096, lr=3e-3, seed=0):
    """Fit the learned Newton guess to recorded samples (n, 5) from newton_samples()."""
    x, y = samples[:, :4], samples[:, 4]
    xm, xs = x.mean(0), x.std(0) + 1e-6
    w0 = mlp_init(seed, xm, xs, float(y.mean()), float(y.std() + 1e-6))
    return mlp_train(w0, x, y, epochs, batch, lr, seed)


# capacity of the static gather buffer of dfd_get_slice_noalloc (DFD_SLICE_SCRATCH_FLOATS)
SLICE_SCRATCH_FLOATS = 1 << 22


class DfdError(RuntimeError):
    def __init__(self, status, msg=""):
        super().__init__(f"{STATUS.get(status, status)}{': ' + msg if msg else ''}")
        self.status = status


class DfdParams(ctypes.Structure):
    _fields_ = [
        ("NX", ctypes.c_int), ("NY", ctypes.c_int), ("NZ", ctypes.c_int), ("NT", ctypes.c_int),
        ("TMAX", ctypes.c_double), ("DT", ctypes.c_double), ("DH", ctypes.c_double),
        ("INPORT_GRID_TYPE", ctypes.c_int), ("INPORT_STRESS_TYPE", ctypes.c_int), ("Friction_type", ctypes.c_int),
        ("EXPORT_TIME_SKIP", ctypes.c_int), ("EXPORT_WAVE_SLICE_X", ctypes.c_int),
        ("EXPORT_WAVE_SLICE_Y", ctypes.c_int), ("EXPORT_WAVE_SLICE_Z", ctypes.c_int),
        ("PML_N", ctypes.c_int), ("PML_velocity", ctypes.c_double), ("PML_bmax", ctypes.c_double),
        ("PML_fc", ctypes.c_double), ("DAMP_N", ctypes.c_int),
        ("mu_s", ctypes.c_double), ("mu_d", ctypes.c_double), ("mu_0", ctypes.c_double), ("Dc", ctypes.c_double),
        ("C0", ctypes.c_double), ("f0", ctypes.c_double), ("V0", ctypes.c_double), ("Vini", ctypes.c_double),
        ("fw", ctypes.c_double), ("L", ctypes.c_double), ("smooth_load_T", ctypes.c_double),
        ("viscosity", ctypes.c_double), ("Fault_grid", ctypes.c_int * 4), ("Asp_grid", ctypes.c_int * 4),
        ("bi_vp1", ctypes.c_double), ("bi_vs1", ctypes.c_double), ("bi_rho1", ctypes.c_double),
        ("bi_vp2", ctypes.c_double), ("bi_vs2", ctypes.c_double), ("bi_rho2", ctypes.c_double),
        ("rupture", ctypes.c_int), ("free_surface", ctypes.c_int), ("use_pml", ctypes.c_int),
        ("use_cerjan", ctypes.c_int), ("normal_refine", ctypes.c_int), ("rs_guess", ctypes.c_int),
        ("OUT", ctypes.c_char * 1024), ("Fault_geometry", ctypes.c_char * 1024),
        ("Fault_init_stress", ctypes.c_char * 1024), ("Media1D", ctypes.c_char * 1024),
        ("TP_n", ctypes.c_int), ("rs_guess_tol", ctypes.c_double), ("slabs_y", ctypes.c_int), ("slab_y", ctypes.c_int),
    ]


# job-file key -> struct field, for keys whose names differ (set_params.cu:137-282 plus the
# reference's compile-time switches as job keys)
_KEYMAP = {"RS_V0": "V0", "RS_Vini": "Vini", "RS_f0": "f0", "RS_fw": "fw", "RS_L": "L", "rho1": "bi_rho1",
           "Rupture": "rupture", "FreeSurface": "free_surface", "usePML": "use_pml", "useCerjan": "use_cerjan",
           "NormalRefine": "normal_refine", "RS_guess": "rs_guess", "RS_guess_tol": "rs_guess_tol"}


def lib():
    """Load libdfd_b200.so (built in-tree); raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"{LIBPATH} is missing: build it with `python -m dynfd3dcuda_b200.build`")
        L = ctypes.CDLL(LIBPATH)
        P, I, V = ctypes.POINTER, ctypes.c_int, ctypes.c_void_p
        sigs = {
            "dfd_params_default": [P(DfdParams)], "dfd_params_load_json": [ctypes.c_char_p, P(DfdParams)],
            "dfd_create": [P(DfdParams), I, P(V)], "dfd_destroy": [V], "dfd_dims": [V, P(I), P(I), P(I)],
            "dfd_load_fault_geometry": [V, V], "dfd_load_media1d": [V, I, V], "dfd_load_fault_init": [V, V],
            "dfd_load_tp_hy": [V, V], "dfd_get_tp_columns": [V, I, V], "dfd_get_fault_table": [V, I, V],
            "dfd_precompute": [V], "dfd_stage": [V, I, I], "dfd_stage_part": [V, I, I, I], "dfd_step": [V, I],
            "dfd_run": [V, I, I],
            "dfd_synchronize": [V], "dfd_get_wave": [V, V], "dfd_set_wave": [V, V], "dfd_get_metric": [V, V],
            "dfd_get_fault": [V, I, V], "dfd_get_slice": [V, I, I, V], "dfd_get_slice_noalloc": [V, I, I, V], "dfd_check_finite": [V],
            "dfd_newton_stats": [V, P(ctypes.c_longlong), P(ctypes.c_longlong)],
            "dfd_output_open": [V, ctypes.c_char_p], "dfd_output_write": [V, I], "dfd_output_close": [V],
            "dfd_set_guess_net": [V, V, I], "dfd_fetch_outputs": [V, V],
            "dfd_run_timed": [V, I, I, P(ctypes.c_float), P(ctypes.c_float), P(ctypes.c_float)],
            "dfd_run_graph_timed": [V, I, I, P(ctypes.c_float)],
            "dfd_interior_stats": [V, P(ctypes.c_float), P(ctypes.c_longlong)],
            "dfd_ens_create": [V, I, P(ctypes.c_void_p)], "dfd_ens_destroy": [V], "dfd_ens_run": [V, I, I],
            "dfd_ens_synchronize": [V], "dfd_ens_run_timed": [V, I, I, P(ctypes.c_float)],
            "dfd_ens_set_chunk": [V, I], "dfd_ens_set_tile_rows": [V, I], "dfd_set_tile_rows": [V, I], "dfd_ens_nodes": [V, P(ctypes.c_longlong)],
            "dfd_newton_record": [V, I, I], "dfd_rs_profile": [V, I, I], "dfd_test_wait_drill": [V, I],
            "dfd_halo_floats": [V, P(ctypes.c_longlong)], "dfd_halo_pack": [V, I, I, V], "dfd_halo_unpack": [V, I, I, V],
            "dfd_rs_solve_stats": [V, P(ctypes.c_longlong), P(ctypes.c_longlong), P(ctypes.c_double),
                                   P(ctypes.c_double)], "dfd_fault_node_ms": [V, P(ctypes.c_float)], "dfd_newton_samples": [V, V, I, P(ctypes.c_int)],
            "dfd_mlp_init": [V, ctypes.c_uint, V, V, ctypes.c_float, ctypes.c_float],
            "dfd_mlp_forward": [V, V, I, V], "dfd_mlp_forward_node": [V, V, I, I, V],
            "dfd_mlp_loss_grad": [V, V, V, I, P(ctypes.c_double), V],
            "dfd_mlp_train": [V, V, I, I, I, ctypes.c_float, ctypes.c_uint, V, V],
        }
        for name, args in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.dfd_error_string.restype = ctypes.c_char_p
        L.dfd_error_string.argtypes = [I]
        L.dfd_last_error.restype = ctypes.c_char_p
        L.dfd_last_error.argtypes = [V]
        _lib = L
    return _lib


def params_struct(job):
    """Reference job dictionary (params.json keys) -> dfd_params, with the reference defaults."""
    L = lib()
    s = DfdParams()
    L.dfd_params_default(ctypes.byref(s))
    for key, val in job.items():
        name = _KEYMAP.get(key, key)
        if name in ("Fault_grid", "Asp_grid"):
            arr = getattr(s, name)
            for i in range(4):
                arr[i] = int(val[i])
        elif name in ("OUT", "Fault_geometry", "Fault_init_stress", "Media1D"):
            setattr(s, name, str(val).encode()[:1023])
        elif any(name == f[0] for f in DfdParams._fields_):
            cur = getattr(s, name)
            setattr(s, name, int(val) if isinstance(cur, int) else float(val))
    # NT = (int)((float)TMAX / (float)DT), single-precision division as the library does
    s.NT = int(np.float32(s.TMAX) / np.float32(s.DT)) if s.DT > 0 else 0
    return s


class Simulation:
    """One rupture simulation resident on one GPU (a dfd_ctx)."""

    def __init__(self, job, fxyz=None, stress=None, layers=None, device=0, precompute=True):
        if isinstance(job, str):
            with open(job) as f:
                job = json.load(f)
        self.job = dict(job)
        self.p = params_struct(self.job)
        L = lib()
        h = ctypes.c_void_p()
        self._check(L.dfd_create(ctypes.byref(self.p), device, ctypes.byref(h)))
        self.h = h
        nx, ny, nz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L.dfd_dims(self.h, ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(nz))
        self.nx, self.ny, self.nz = nx.value, ny.value, nz.value
        # NY: the columns this context holds (NY / slabs_y for a slab of a decomposed domain)
        self.NX, self.NY, self.NZ = self.p.NX, self.ny - 6, self.p.NZ
        if fxyz is not None:
            a = np.ascontiguousarray(fxyz, np.float32)
            self._check(L.dfd_load_fault_geometry(self.h, a.ctypes.data))
        if stress is not None:
            a = np.ascontiguousarray(stress, np.float32)
            self._check(L.dfd_load_fault_init(self.h, a[:15].ctypes.data))
            if a.shape[0] > 15:  # TP_hy, the 16th variable of the init file (Friction_type 3)
                hy = np.ascontiguousarray(a[15])
                self._check(L.dfd_load_tp_hy(self.h, hy.ctypes.data))
        if layers is not None:
            a = np.ascontiguousarray(layers, np.float32)
            self._check(L.dfd_load_media1d(self.h, a.shape[0], a.ctypes.data))
        if precompute:
            self.precompute()

    def _check(self, r):
        if r:
            msg = ""
            if getattr(self, "h", None):
                msg = (lib().dfd_last_error(self.h) or b"").decode()
            raise DfdError(r, msg)

    def close(self):
        if getattr(self, "h", None):
            lib().dfd_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def precompute(self):
        self._check(lib().dfd_precompute(self.h))

    def stage(self, it, irk):
        self._check(lib().dfd_stage(self.h, it, irk))

    def stage_part(self, it, irk, part):
        """Part 0 (fault trial), 1 (volume) or 2 (fault band) of stage irk of step it."""
        self._check(lib().dfd_stage_part(self.h, it, irk, part))

    def step(self, it):
        self._check(lib().dfd_step(self.h, it))

    def run(self, it0, nsteps):
        self._check(lib().dfd_run(self.h, it0, nsteps))

    def synchronize(self):
        self._check(lib().dfd_synchronize(self.h))

    def wave(self):
        out = np.empty((9, self.nx, self.nz, self.ny), np.float32)
        self._check(lib().dfd_get_wave(self.h, out.ctypes.data))
        return out

    def set_wave(self, w):
        a = np.ascontiguousarray(w, np.float32)
        assert a.size == 9 * self.nx * self.ny * self.nz
        self._check(lib().dfd_set_wave(self.h, a.ctypes.data))

    def metric(self):
        out = np.empty((13, self.nx, self.nz, self.ny), np.float32)
        self._check(lib().dfd_get_metric(self.h, out.ctypes.data))
        return out

    def fault(self, name):
        f = FIELDS.index(name)
        if name == "split":
            out = np.empty((9, 2, self.nz, self.ny), np.float32)
        elif name == "T1":
            out = np.empty((3, 7, self.nz, self.ny), np.float32)
        elif name == "hT1":
            out = np.empty((3, self.nz, self.ny), np.float32)
        else:
            out = np.empty((self.NZ, self.NY), np.float32)
        self._check(lib().dfd_get_fault(self.h, f, out.ctypes.data))
        return out

    def fault_table(self, name):
        """A split-node coefficient table by its reference name (TABLES): (nz, ny, 9) per
        fault node, (ny, 9) on the free-surface row, (nz, ny, 3) for vec_n/vec_s1/vec_s2."""
        t = TABLES.index(name)
        if name.startswith("vec_"):
            out = np.empty((self.nz, self.ny, 3), np.float32)
        elif t >= TABLES.index("matVx2Vz1"):
            out = np.empty((self.ny, 9), np.float32)
        else:
            out = np.empty((self.nz, self.ny, 9), np.float32)
        self._check(lib().dfd_get_fault_table(self.h, t, out.ctypes.data))
        return out

    def tp_columns(self, name):
        """Thermal-pressurisation columns "TP_T" or "TP_P", (TP_n, NZ, NY), point 0 on the fault."""
        out = np.empty((self.p.TP_n, self.NZ, self.NY), np.float32)
        self._check(lib().dfd_get_tp_columns(self.h, ("TP_T", "TP_P").index(name), out.ctypes.data))
        return out

    def slice(self, axis, index):
        na = self.NZ if axis == 0 else self.NX
        nb = self.NZ if axis == 1 else self.NY
        out = np.empty((3, na, nb), np.float32)
        self._check(lib().dfd_get_slice(self.h, axis, index, out.ctypes.data))
        return out

    def slice_noalloc(self, axis, index):
        """Same as slice(), gathered in the library's static device buffer (no allocation)."""
        na = self.NZ if axis == 0 else self.NX
        nb = self.NZ if axis == 1 else self.NY
        out = np.empty((3, na, nb), np.float32)
        self._check(lib().dfd_get_slice_noalloc(self.h, axis, index, out.ctypes.data))
        return out

    def check_finite(self):
        self._check(lib().dfd_check_finite(self.h))

    def newton_stats(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(lib().dfd_newton_stats(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def halo_floats(self):
        """Floats of one halo message (dfd_halo_floats)."""
        n = ctypes.c_longlong()
        self._check(lib().dfd_halo_floats(self.h, ctypes.byref(n)))
        return n.value

    def halo_pack(self, what, side, device_ptr):
        """Gather the leaving columns of side 0 (low y) or 1 (high y) into device memory;
        what = 0..3 (the input of that RK stage) or HALO_SETUP."""
        self._check(lib().dfd_halo_pack(self.h, what, side, device_ptr))

    def halo_unpack(self, what, side, device_ptr):
        """Scatter a neighbour's message into the ghost columns of side 0 or 1."""
        self._check(lib().dfd_halo_unpack(self.h, what, side, device_ptr))

    def test_wait_drill(self, on=True):
        """Test hook: the interior kernel issues no copies, so its bounded waits run out."""
        self._check(lib().dfd_test_wait_drill(self.h, int(on)))

    def rs_profile(self, timing=True, judge=False):
        """Switch the rate-and-state solve measurement aids (solve timing, plain-solve judge)."""
        self._check(lib().dfd_rs_profile(self.h, int(timing), int(judge)))

    def rs_solve_stats(self):
        """(accepted learned guesses, fallbacks to the plain solve, mean clock cycles of a timed
        solve, judge's largest relative difference)."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        c, d = ctypes.c_double(), ctypes.c_double()
        self._check(lib().dfd_rs_solve_stats(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                             ctypes.byref(d)))
        return a.value, b.value, c.value, d.value

    def fetch_outputs(self, host_ptr):
        """Enqueue the copy of the (8, NZ, NY) per-step outputs into host memory at host_ptr."""
        self._check(lib().dfd_fetch_outputs(self.h, host_ptr))

    def run_timed(self, it0, nsteps):
        """Run nsteps stage by stage; returns (total_ms, volume_kernel_ms, other_ms) from CUDA events."""
        t, v, f = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        self._check(lib().dfd_run_timed(self.h, it0, nsteps, ctypes.byref(t), ctypes.byref(v), ctypes.byref(f)))
        return t.value, v.value, f.value

    def run_graph_timed(self, it0, nsteps):
        """Replay nsteps steps from the CUDA graphs (all built beforehand); device time in ms."""
        ms = ctypes.c_float()
        self._check(lib().dfd_run_graph_timed(self.h, it0, nsteps, ctypes.byref(ms)))
        return ms.value

    def interior_stats(self):
        """(ms, nodes): interior-kernel device time of the last run_timed and nodes per stage."""
        ms, nodes = ctypes.c_float(), ctypes.c_longlong()
        self._check(lib().dfd_interior_stats(self.h, ctypes.byref(ms), ctypes.byref(nodes)))
        return ms.value, nodes.value

    def set_guess_net(self, w):
        """Load MLP weights (MLP_PARAMS floats) and use the learned Newton guess; None: plain guess."""
        if w is None:
            self._check(lib().dfd_set_guess_net(self.h, None, 0))
            return
        a = np.ascontiguousarray(w, np.float32).ravel()
        self._check(lib().dfd_set_guess_net(self.h, a.ctypes.data, a.size))

    def set_tile_rows(self, rows):
        """Rows of the interior kernel's tiles: 8 (one CTA per SM, the default) or 4 (two
        CTAs per SM); the same results either way."""
        self._check(lib().dfd_set_tile_rows(self.h, int(rows)))

    def newton_record(self, capacity, every=1):
        """Record (psi/a, log10 Vhat, log10 coef, a, x* residual) of one in `every` converged
        plain Newton solves, up to capacity samples (0 stops recording)."""
        self._check(lib().dfd_newton_record(self.h, int(capacity), int(every)))

    def fault_node_ms(self):
        """Fault node kernel device time of the last run_timed (ms, all stages)."""
        ms = ctypes.c_float()
        self._check(lib().dfd_fault_node_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def newton_samples(self, max_samples):
        out = np.empty((max(int(max_samples), 1), 5), np.float32)
        n = ctypes.c_int()
        self._check(lib().dfd_newton_samples(self.h, out.ctypes.data, int(max_samples), ctypes.byref(n)))
        return out[:n.value].copy()

    def output_open(self, outdir):
        self._check(lib().dfd_output_open(self.h, outdir.encode()))

    def output_write(self, it_skip):
        self._check(lib().dfd_output_write(self.h, it_skip))

    def output_close(self):
        self._check(lib().dfd_output_close(self.h))
