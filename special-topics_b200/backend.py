"""The B200 backend behind the reference's backend contract.

Mirrors js_fdtd/src/backends/CONTRACT.md:104-137 and the CUDA backend driver
js_fdtd/src/backends/cuda/cudaBackend.js:165-306: an object with ``name``,
``is_available()`` (never raises) and ``run(problem)``, a generator that
advances the whole time loop on the GPU, yields a progress snapshot every
``batch_size`` steps and on the last step, and leaves the port traces and
far-field accumulators filled in (``Engine.voltages()`` ... ``farfield()``).

``Engine`` is the handle-level API: it uploads a ``scenario.Problem`` through
the C ABI (include/fdtd_b200.h) and exposes the device state for checks.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Iterator

import numpy as np

from . import _native as N
from .scenario import COEFF_ORDER, FF_NAMES, Problem
from .tables import COMPONENTS, build_tables, check_source_outside_cpml

PRECISIONS = {"f64": N.PREC_F64, "f32": N.PREC_F32, "f32-table": N.PREC_F32_TABLE}
FIELD_IDS = {"Hx": 0, "Hy": 1, "Hz": 2, "Ex": 3, "Ey": 4, "Ez": 5}


class Engine:
    """One problem resident on one GPU."""

    def __init__(self, problem: Problem, precision: str = "f64", device: int = 0, host_tables: bool = False,
                 dft_accumulator: str = "f64", dft_block: int = 0, x_wall: bool | None = None):
        """host_tables=True builds an FP32-table problem's ids with numpy
        (tables.build_tables, needs per-cell material arrays) instead of on the
        device (fdtd_ctx_build_material).  dft_accumulator "kahan-f32" keeps an
        FP32 problem's far-field accumulators as compensated FP32 pairs; dft_block
        > 0 accumulates the surface DFT once per that many steps (FP32).
        x_wall: None keeps the precision's default (FP64: the reference's reads
        past Hz/Hy at i = nx; FP32: Ey, Ez at i = nx held at zero), True / False
        forces the wall / the reference's reads (fdtd_ctx_set_x_wall)."""
        if dft_accumulator not in ("f64", "kahan-f32"):
            raise ValueError("dft_accumulator must be 'f64' or 'kahan-f32'")
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        L = N.lib()
        self.problem = problem
        self.precision = precision
        self.host_tables = host_tables
        g = problem.grid
        cfg = N.FdtdConfig(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.dt, g.numberOfTimeSteps,
                           PRECISIONS[precision], device)
        h = C.c_void_p()
        N.check(L.fdtd_create(C.byref(cfg), C.byref(h)))
        self._h = h
        try:
            self._upload()
            if dft_accumulator == "kahan-f32":
                N.check(L.fdtd_ctx_set_dft_accumulator(h, 1))
            if dft_block:
                N.check(L.fdtd_ctx_set_dft_block(h, int(dft_block)))
            if x_wall is not None:
                N.check(L.fdtd_ctx_set_x_wall(h, int(bool(x_wall))))
        except Exception:
            self.close()
            raise

    # -- upload -------------------------------------------------------------
    def _upload(self) -> None:
        L, p, h = N.lib(), self.problem, self._h
        table = self.precision == "f32-table"
        if table and self.host_tables:
            for comp_id, (ids, tab) in enumerate(build_tables(p)[c] for c in COMPONENTS):
                N.check(L.fdtd_ctx_upload_material(h, comp_id, ids.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                                   ids.size, N.dptr(tab.ravel()), tab.shape[0]))
        elif table or (self.precision == "f64" and not p.coeffs):
            # FP64 problems built without per-cell arrays get them on the device
            self._build_tables_on_device()
        else:
            for w, name in enumerate(COEFF_ORDER):
                a = np.ascontiguousarray(p.coeffs[name], dtype=np.float64)
                N.check(L.fdtd_ctx_upload_coeff(h, w, N.dptr(a), a.size))
        for fid, f in enumerate(p.cpml):
            if f is None:
                continue
            prof = [np.ascontiguousarray(x, dtype=np.float64)
                    for x in (f.b_e, f.a_e, f.b_m, f.a_m, f.kappa_e, f.kappa_m)]
            args = []
            for cp in (f.cpsi if (not table and f.cpsi is not None) else [None] * 4):
                if cp is None:
                    args += [None, 0]
                else:
                    cp = np.ascontiguousarray(cp, dtype=np.float64)
                    args += [N.dptr(cp), cp.size]
            N.check(L.fdtd_ctx_upload_cpml(h, fid, f.nc, *[N.dptr(x) for x in prof], *args, f.m_start, f.e_start))
        for vs in p.voltage_sources:
            fi = np.ascontiguousarray(vs.field_indices, dtype=np.int32)
            cs = np.ascontiguousarray(vs.coef, dtype=np.float64)
            wv = np.ascontiguousarray(vs.voltage_per_e_field, dtype=np.float64)
            N.check(L.fdtd_ctx_add_vsource(h, vs.axis, N.iptr(fi), N.dptr(cs), fi.size, N.dptr(wv), wv.size))
        for sv in p.sampled_voltages:
            fi = np.ascontiguousarray(sv.field_indices, dtype=np.int32)
            N.check(L.fdtd_ctx_add_svoltage(h, sv.axis, N.iptr(fi), fi.size, sv.Csvf))
        for si in p.sampled_currents:
            comp = np.ascontiguousarray(si.comp, dtype=np.int32)
            idx = np.ascontiguousarray(si.idx, dtype=np.int32)
            w = np.ascontiguousarray(si.w, dtype=np.float64)
            N.check(L.fdtd_ctx_add_scurrent(h, N.iptr(comp), N.iptr(idx), N.dptr(w), comp.size))
        ff = p.farfield
        if ff is not None and ff.nFreq > 0:
            fr = np.ascontiguousarray(ff.frequencies, dtype=np.float64)
            N.check(L.fdtd_ctx_setup_farfield(h, fr.size, N.dptr(fr), ff.li, ff.lj, ff.lk, ff.ui, ff.uj, ff.uk))

    def _build_tables_on_device(self) -> None:
        """Material tables (FP32-table), or the 18 per-cell FP64 coefficient
        arrays, from the problem's material grid on the device, then the
        lumped-source cells' own triples.  (For FP64 the CPML kappa division
        follows when the faces are uploaded without CPsi.)"""
        L, p, h = N.lib(), self.problem, self._h
        mat = np.ascontiguousarray(p.meta["material_grid"], dtype=np.uint8).ravel()
        props = np.ascontiguousarray(p.meta["material_props"], dtype=np.float64)
        plates = p.meta["plates"]
        pl = np.ascontiguousarray(np.array([b[:7] for b in plates], dtype=np.int32).reshape(-1))
        ps = np.ascontiguousarray(np.array([b[7] for b in plates], dtype=np.float64))
        N.check(L.fdtd_ctx_build_material(h, mat.ctypes.data_as(C.POINTER(C.c_ubyte)), mat.size, props.shape[0],
                                          N.dptr(props.reshape(-1)), len(plates), N.iptr(pl), N.dptr(ps)))
        for vs in p.voltage_sources:
            check_source_outside_cpml(vs, p)
            fi = np.ascontiguousarray(vs.field_indices, dtype=np.int32)
            trip = np.ascontiguousarray(vs.override, dtype=np.float64).reshape(-1)
            N.check(L.fdtd_ctx_override_material(h, vs.axis, N.iptr(fi), N.dptr(trip), fi.size))

    @property
    def x_wall(self) -> bool:
        w = C.c_int()
        N.check(N.lib().fdtd_ctx_get_x_wall(self._h, C.byref(w)))
        return bool(w.value)

    @x_wall.setter
    def x_wall(self, wall: bool) -> None:
        N.check(N.lib().fdtd_ctx_set_x_wall(self._h, int(bool(wall))))

    def material(self, comp: str) -> tuple[np.ndarray, np.ndarray]:
        """(ids, FP64 table rows x 3) of a table problem's component."""
        n = int(np.prod(self.problem.grid.shapes[comp]))
        ids = np.zeros(n, dtype=np.uint8)
        tab = np.zeros(256 * 3)
        rows = C.c_int()
        N.check(N.lib().fdtd_ctx_read_material(self._h, COMPONENTS.index(comp), ids.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                               n, N.dptr(tab), C.byref(rows)))
        return ids, tab[:3 * rows.value].reshape(-1, 3)

    # -- stepping -------------------------------------------------------------
    @property
    def step(self) -> int:
        return N.lib().fdtd_ctx_step(self._h)

    def run(self, count: int) -> None:
        N.check(N.lib().fdtd_ctx_run(self._h, int(count)))

    def run_timed(self, count: int) -> float:
        """Runs `count` steps; returns their device time in ms (CUDA events on the engine's stream)."""
        ms = C.c_float()
        N.check(N.lib().fdtd_ctx_run_timed(self._h, int(count), C.byref(ms)))
        return ms.value

    def profile_kernels(self, count: int) -> dict:
        """Mean device ms of each kernel over `count` steps run one launch at a time."""
        out = np.zeros(4)
        N.check(N.lib().fdtd_ctx_profile_kernels(self._h, int(count), N.dptr(out)))
        return dict(zip(("h", "mid", "e", "epilogue"), out.tolist()))

    def status(self) -> tuple[int, int]:
        code, step = C.c_int(), C.c_int()
        N.check(N.lib().fdtd_status(self._h, C.byref(code), C.byref(step)))
        return code.value, step.value

    # -- readback -------------------------------------------------------------
    def _trace(self, kind: int, q: int, n: int | None) -> np.ndarray:
        n = self.step if n is None else n
        out = np.zeros(n)
        N.check(N.lib().fdtd_ctx_read_trace(self._h, kind, q, N.dptr(out), n))
        return out

    def voltages(self, n: int | None = None) -> list:
        return [self._trace(0, q, n) for q in range(len(self.problem.sampled_voltages))]

    def currents(self, n: int | None = None) -> list:
        return [self._trace(1, q, n) for q in range(len(self.problem.sampled_currents))]

    def field(self, name: str) -> np.ndarray:
        shape = self.problem.grid.shapes[name]
        out = np.zeros(int(np.prod(shape)))
        N.check(N.lib().fdtd_ctx_read_field(self._h, FIELD_IDS[name], N.dptr(out), out.size))
        return out

    def psi(self, face: int, slot: int, n: int) -> np.ndarray:
        out = np.zeros(n)
        N.check(N.lib().fdtd_ctx_read_psi(self._h, face, slot, N.dptr(out), n))
        return out

    def farfield(self) -> dict[str, tuple[np.ndarray, np.ndarray]]:
        ff = self.problem.farfield
        if ff is None:
            return {}
        ni, nj, nk = ff.ui - ff.li, ff.uj - ff.lj, ff.uk - ff.lk
        sizes = (nj * nk, ni * nk, ni * nj)
        out = {}
        for a, name in enumerate(FF_NAMES):
            n = ff.nFreq * sizes[(a % 12) // 4]
            re, im = np.empty(n), np.empty(n)      # every value is overwritten
            N.check(N.lib().fdtd_ctx_read_farfield(self._h, a, N.dptr(re), N.dptr(im), n))
            out[name] = (re, im)
        return out

    def save_state(self) -> bytes:
        """The evolving state (fields, Psi, traces, accumulators, step) as bytes."""
        n = C.c_longlong()
        N.check(N.lib().fdtd_ctx_state_size(self._h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        N.check(N.lib().fdtd_ctx_save_state(self._h, buf, n.value))
        return buf.raw

    def load_state(self, state: bytes) -> None:
        """Restores a state saved from an engine of the same problem."""
        buf = C.create_string_buffer(state, len(state))
        N.check(N.lib().fdtd_ctx_load_state(self._h, buf, len(state)))

    def farfield_post(self, theta, phi):
        """Radiated power [nFreq] and directivity D_theta, D_phi [nFreq, nang]
        computed on the device from the accumulators (farfield.js:257-607)."""
        theta = np.ascontiguousarray(theta, dtype=np.float64).ravel()
        phi = np.ascontiguousarray(phi, dtype=np.float64).ravel()
        if theta.shape != phi.shape:
            raise ValueError("theta and phi must have the same length")
        nf = self.problem.farfield.nFreq if self.problem.farfield is not None else 0
        radp = np.zeros(max(nf, 1))
        dth = np.zeros((max(nf, 1), theta.size))
        dph = np.zeros((max(nf, 1), theta.size))
        N.check(N.lib().fdtd_ctx_farfield_post(self._h, N.dptr(theta), N.dptr(phi), theta.size, N.dptr(radp),
                                               N.dptr(dth), N.dptr(dph)))
        return radp[:nf], dth[:nf], dph[:nf]

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            N.lib().fdtd_free(h)
        self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Engines of one precision on one device advanced together
    (fdtd_batch_* in include/fdtd_b200.h).  streams = 0: every step is four
    launches for the whole batch over a tile list, or, with per_launch = P > 0,
    H and E launches that each carry P members' parameter blocks as their
    kernel parameter (grouped mode); streams = S > 0: each member's own step
    kernels on S worker streams in one graph.  The engines stay usable for
    readback and must outlive the batch."""

    def __init__(self, engines: list, chunk: int = 8, rows: int = 4, prefetch: int = 1, group: int = 0,
                 streams: int = 0):
        if not engines:
            raise ValueError("a batch needs at least one engine")
        self.engines = list(engines)
        arr = (C.c_void_p * len(self.engines))(*[e._h.value for e in self.engines])
        h = C.c_void_p()
        N.check(N.lib().fdtd_batch_create(arr, len(self.engines), C.byref(h)))
        self._h = h
        self.set_tiling(chunk, rows, prefetch, group, streams)

    def set_tiling(self, chunk: int, rows: int, prefetch: int = 1, group: int = 0, streams: int | None = None,
                   width: int | None = None, per_launch: int | None = None) -> None:
        """Launch shape (see fdtd_batch_set_tiling) and, when given, the
        member-kernel worker stream count (fdtd_batch_set_streams), the
        block width along k (fdtd_batch_set_block_width) and the members per
        grouped launch (fdtd_batch_set_members_per_launch)."""
        N.check(N.lib().fdtd_batch_set_tiling(self._h, int(chunk), int(rows), int(prefetch), int(group)))
        if streams is not None:
            N.check(N.lib().fdtd_batch_set_streams(self._h, int(streams)))
        if width is not None:
            N.check(N.lib().fdtd_batch_set_block_width(self._h, int(width)))
        if per_launch is not None:
            N.check(N.lib().fdtd_batch_set_members_per_launch(self._h, int(per_launch)))

    def set_shape(self, shape: dict) -> None:
        """set_tiling from a dict as tiling() returns it ("streams" and
        "width" optional)."""
        self.set_tiling(shape["chunk"], shape["rows"], shape.get("prefetch", 1), shape.get("group", 0),
                        shape.get("streams", 0), shape.get("width", 32), shape.get("per_launch", 0))

    def tiling(self) -> dict:
        v = [C.c_int() for _ in range(7)]
        N.check(N.lib().fdtd_batch_get_tiling(self._h, *[C.byref(x) for x in v[:4]]))
        N.check(N.lib().fdtd_batch_get_streams(self._h, C.byref(v[4])))
        N.check(N.lib().fdtd_batch_get_block_width(self._h, C.byref(v[5])))
        N.check(N.lib().fdtd_batch_get_members_per_launch(self._h, C.byref(v[6])))
        return dict(zip(("chunk", "rows", "prefetch", "group", "streams", "width", "per_launch"),
                        [x.value for x in v]))

    @property
    def cells(self) -> int:
        return sum(e.problem.grid.nx * e.problem.grid.ny * e.problem.grid.nz for e in self.engines)

    @property
    def step(self) -> int:
        return self.engines[0].step

    def run(self, count: int) -> None:
        N.check(N.lib().fdtd_batch_run(self._h, int(count)))

    def run_timed(self, count: int) -> float:
        ms = C.c_float()
        N.check(N.lib().fdtd_batch_run_timed(self._h, int(count), C.byref(ms)))
        return ms.value

    def profile_kernels(self, count: int) -> dict:
        out = np.zeros(4)
        N.check(N.lib().fdtd_batch_profile_kernels(self._h, int(count), N.dptr(out)))
        return dict(zip(("h", "mid", "e", "epilogue"), out.tolist()))

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            N.lib().fdtd_batch_free(h)
        self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class B200Backend:
    """Backend object of the reference's registry contract (CONTRACT.md:121-137)."""

    name = "b200"

    def __init__(self, precision: str = "f64", device: int = 0):
        self.precision = precision
        self.device = device
        self.engine: Engine | None = None

    def is_available(self) -> bool:
        try:
            return N.device_count() > 0
        except Exception:
            return False

    def meta(self) -> dict:
        return {"name": self.name, "precision": self.precision, "farfield": "device"}

    def run(self, problem: Problem, batch_size: int = 50) -> Iterator[dict]:
        g = problem.grid
        total = g.numberOfTimeSteps
        eng = Engine(problem, self.precision, self.device)
        self.engine = eng
        t0 = time.time()
        ts = 0
        while ts < total:
            n = min(batch_size, total - ts)
            eng.run(n)
            ts += n
            v = None
            if problem.sampled_voltages:
                v = float(eng._trace(0, 0, ts)[ts - 1])
            yield {"step": ts, "total": total, "elapsed": time.time() - t0,
                   "percent": f"{ts / total * 100:.1f}", "voltage": v,
                   "time_ns": (ts - 1 + 0.5) * g.dt * 1e9, "backend": self.name}
