"""rmt3d_b200: B200 implementation of RMT3D's per-timestep Eulerian FSI update.

Host-side mirror of the reference's seam for this path:

* :class:`Scene` stands in for ``fluid_3d`` (F3D_Source/fluid_3d.hh:37-467):
  ``initialize``, ``set_dt``, ``init_iter``, ``step_forward`` keep the
  reference's names, argument meaning and integer return codes.
* :class:`Stepper` stands in for ``stepper`` (Sim/stepper.hh:22-376): dt
  fitting to frames and the frame/step loop with ``stop_short``.
* :func:`run_sim` is the ``run_sim`` driver sequence (Execs/run_sim.cc:39-141).

All work runs in the CUDA library ``librmt3d_gpu.so`` through the C ABI of
include/rmt3d_gpu.h; there is no CPU path.
"""
import ctypes
import os

import numpy as np

from . import _lib
from ._lib import FP64, MIXED, MIXED_BULK32, PROJECTION_ERR, REFMAP_UPDATE_ERR, STEADY_SOLN_EXIT  # noqa: F401
from ._lib import OK as NORMAL_EXIT
from ._lib import RMT3DError, SceneDesc

# write_params::default_names (IO/write_params.cc:3): slice output types 0-21
OUTPUT_NAMES = ["vx", "vy", "vz", "wx", "wy", "wz", "w", "p", "phi", "X", "Y", "Z", "OID", "LID", "pr_phi",
                "pr_X", "pr_Y", "pr_Z", "div_u", "div_eu", "rho", "J"]

FIELD_INDEX = {"u": 0, "v": 1, "w": 2, "p": 3, "dp": 4, "q": 5, "du": 6, "dv": 7, "dw": 8}
for _f in range(6):
    for _c in range(3):
        FIELD_INDEX["fvel%d%d" % (_f, _c)] = 9 + 3 * _f + _c
for _F in range(3):
    for _c in range(3):
        FIELD_INDEX["sigma%d%d" % (_F, _c)] = 27 + 3 * _F + _c


def lib():
    return _lib.load()


def desc_from_cfg(path):
    """sim_params(cfg) (Sim/sim_params.cc:10-410) into a SceneDesc."""
    L = lib()
    d = SceneDesc()
    _lib.check(L.rmt3d_desc_from_cfg(str(path).encode(), ctypes.byref(d)))
    return d


def desc_defaults():
    L = lib()
    d = SceneDesc()
    _lib.check(L.rmt3d_desc_defaults(ctypes.byref(d)))
    return d


def stepper_dt(desc, dt_reg):
    """stepper dt fit (Sim/stepper.hh:220-225) -> (dt, steps per frame)."""
    L = lib()
    dt = ctypes.c_double()
    steps = ctypes.c_int()
    _lib.check(L.rmt3d_stepper_dt(ctypes.byref(desc), dt_reg, ctypes.byref(dt), ctypes.byref(steps)))
    return dt.value, steps.value


class Scene:
    """One simulation scene on the current CUDA device (``fluid_3d``)."""

    def __init__(self, desc, stream=None):
        L = lib()
        self.desc = desc
        h = ctypes.c_void_p()
        st = ctypes.c_void_p(stream if stream is not None else 0)
        _lib.check(L.rmt3d_scene_create(ctypes.byref(desc), st, ctypes.byref(h)))
        self._h = h
        dims = (ctypes.c_int * 6)()
        _lib.check(L.rmt3d_get_dims(h, dims))
        self.sm4, self.sn4, self.so4, self.fm, self.fn, self.fo = list(dims)
        self.ncell = self.sm4 * self.sn4 * self.so4

    @classmethod
    def from_cfg(cls, path, **overrides):
        d = desc_from_cfg(path)
        for k, v in overrides.items():
            setattr(d, k, v)
        return cls(d)

    # -- the fluid_3d members the stepper and run_sim use -------------------
    def initialize(self):
        """Returns init_err: 0 restarted from the descriptor's checkpoint
        (run.chk_num > 0), 1 started from scratch (fluid_3d.cc:192-233)."""
        _lib.check(lib().rmt3d_initialize(self._h))
        return int(self.scalar(13))

    def set_dt(self, dt):
        _lib.check(lib().rmt3d_set_dt(self._h, dt))

    def init_iter(self, init_err=None):
        """Pressure pre-iterations when the last initialize started from
        scratch, then the stress of the current state; init_err, when given,
        must be that initialize's result."""
        if init_err is not None and int(init_err) != int(self.scalar(13)):
            raise ValueError("init_err differs from the last initialize's result")
        _lib.check(lib().rmt3d_init_iter(self._h))

    def write_chk_pt(self, snum, fnum, chk_dirname, compress=True):
        """Checkpoint in the reference's format (fluid_3d_chk_pt.cc:3-72)."""
        _lib.check(lib().rmt3d_write_chk_pt(self._h, int(snum), int(fnum), str(chk_dirname).encode(),
                                            int(bool(compress))))

    def read_chk_pt(self, chk_dirname):
        """Restart from a checkpoint directory (fluid_3d_chk_pt.cc:74-163);
        returns the reference's status: 0 read, 1 file missing, 2 file empty."""
        st = ctypes.c_int()
        _lib.check(lib().rmt3d_read_chk_pt(self._h, str(chk_dirname).encode(), ctypes.byref(st)))
        return st.value

    def prepare(self):
        _lib.check(lib().rmt3d_prepare(self._h))

    def step_forward(self, debug=0):
        st = ctypes.c_int()
        _lib.check(lib().rmt3d_step(self._h, debug, ctypes.byref(st)))
        return st.value

    def step_phases(self, last_phase):
        """The first `last_phase` phase groups of one step (inspection)."""
        st = ctypes.c_int()
        _lib.check(lib().rmt3d_step_phases(self._h, last_phase, ctypes.byref(st)))
        return st.value

    def macro(self):
        """The frame diagnostics of macro.dat / centroid.dat (MacroData)."""
        m = _lib.MacroData()
        _lib.check(lib().rmt3d_macro(self._h, ctypes.byref(m)))
        return m

    def tracers(self):
        """Tracer coordinates by id as an (ntracers, 3) float32 array
        (0 0 0 for a lost tracer); empty when the scene has none."""
        n = ctypes.c_int()
        _lib.check(lib().rmt3d_tracer_positions(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 3), dtype=np.float32)
        if n.value:
            _lib.check(lib().rmt3d_tracer_positions(self._h, out.ctypes.data_as(ctypes.c_void_p), n.value,
                                                    ctypes.byref(n)))
        return out

    def place_tracers(self, xyz):
        """Place every tracer at the given coordinates ((ntracers, 3))."""
        a = np.ascontiguousarray(xyz, dtype=np.float64)
        _lib.check(lib().rmt3d_tracer_place(self._h, a.ctypes.data_as(ctypes.c_void_p), a.shape[0]))

    def write_tracers(self, filename, binary=True):
        """tracers::print: binary or text tracer file."""
        _lib.check(lib().rmt3d_write_tracers(self._h, str(filename).encode(), int(bool(binary))))

    def slice(self, otype, dim, point, obj_id=-1):
        """fluid_3d::slice: the global slice array, shape (d2, d1)."""
        d1, d2 = ctypes.c_int(), ctypes.c_int()
        _lib.check(lib().rmt3d_slice(self._h, otype, dim, point, obj_id, None, ctypes.byref(d1), ctypes.byref(d2)))
        out = np.empty(d1.value * d2.value, dtype=np.float64)
        _lib.check(lib().rmt3d_slice(self._h, otype, dim, point, obj_id, out.ctypes.data_as(ctypes.c_void_p),
                                     ctypes.byref(d1), ctypes.byref(d2)))
        return out.reshape(d2.value, d1.value)

    def write_slice(self, otype, dim, point, obj_id, fmt, filename):
        """fluid_3d::write_slice in format 0 (matrix), 1 (text) or 2 (gnuplot)."""
        _lib.check(lib().rmt3d_write_slice(self._h, otype, dim, point, obj_id, fmt, str(filename).encode()))

    def export_reference(self):
        """State in the reference's AoS layout: (fields, refmaps, ext_index, ext_maps)."""
        from .layout import FIELD_DT, REFMAP_DT
        fields = np.zeros(self.ncell, dtype=FIELD_DT)
        rm = np.zeros(self.ncell, dtype=REFMAP_DT)
        n = ctypes.c_int()
        _lib.check(lib().rmt3d_export_reference(self._h, fields.ctypes.data_as(ctypes.c_void_p),
                                                rm.ctypes.data_as(ctypes.c_void_p), None, None, 0,
                                                ctypes.byref(n)))
        idx = np.zeros(max(n.value, 1), dtype=np.int32)
        ext = np.zeros(max(n.value, 1), dtype=REFMAP_DT)
        _lib.check(lib().rmt3d_export_reference(self._h, None, None, idx.ctypes.data_as(ctypes.c_void_p),
                                                ext.ctypes.data_as(ctypes.c_void_p), n.value, ctypes.byref(n)))
        return fields, rm, idx[:n.value], ext[:n.value]

    def run(self, nsteps):
        st = ctypes.c_int()
        _lib.check(lib().rmt3d_run(self._h, nsteps, ctypes.byref(st)))
        return st.value

    def sync(self):
        _lib.check(lib().rmt3d_sync(self._h))

    # -- state access ---------------------------------------------------------
    def scalar(self, which):
        v = ctypes.c_double()
        _lib.check(lib().rmt3d_get_scalar(self._h, which, ctypes.byref(v)))
        return v.value

    @property
    def dt(self):
        return self.scalar(0)

    @property
    def time(self):
        return self.scalar(1)

    @property
    def dt_reg(self):
        return self.scalar(2)

    def field(self, name):
        """Field over the ghosted box as an array of shape (so+4, sn+4, sm+4)."""
        out = np.empty(self.ncell, dtype=np.float64)
        idx = FIELD_INDEX[name] if isinstance(name, str) else int(name)
        _lib.check(lib().rmt3d_get_field(self._h, idx, out.ctypes.data_as(ctypes.c_void_p)))
        return out.reshape(self.so4, self.sn4, self.sm4)

    def refmap(self, obj=0):
        code = np.empty(self.ncell, dtype=np.int32)
        x = np.empty(3 * self.ncell, dtype=np.float64)
        xp = np.empty(3 * self.ncell, dtype=np.float64)
        _lib.check(lib().rmt3d_get_refmap(self._h, obj, code.ctypes.data_as(ctypes.c_void_p),
                                          x.ctypes.data_as(ctypes.c_void_p), xp.ctypes.data_as(ctypes.c_void_p)))
        shp = (self.so4, self.sn4, self.sm4)
        return code.reshape(shp), x.reshape((3,) + shp), xp.reshape((3,) + shp)

    def import_reference(self, field_aos, refmap_aos, ext_index, ext_maps, dt, time):
        fa = np.ascontiguousarray(field_aos)
        ra = np.ascontiguousarray(refmap_aos) if refmap_aos is not None else None
        ei = np.ascontiguousarray(ext_index, dtype=np.int32)
        em = np.ascontiguousarray(ext_maps)
        _lib.check(lib().rmt3d_import_reference(
            self._h, fa.ctypes.data_as(ctypes.c_void_p),
            ra.ctypes.data_as(ctypes.c_void_p) if ra is not None else None,
            ei.ctypes.data_as(ctypes.c_void_p), em.ctypes.data_as(ctypes.c_void_p), len(ei), dt, time))

    def diag(self, kind=0):
        """0 div_u, 1 solid volume, 2-4 solid centroid, 5 total and 6 maximum
        deviation of det F from 1."""
        v = ctypes.c_double()
        _lib.check(lib().rmt3d_diag(self._h, kind, ctypes.byref(v)))
        return v.value

    def profile_kernel(self, kernel, max_launches=100000):
        """Time launches of one kernel class (0 FEM GS fine level, 1 MAC RB fine level, -1 off)."""
        _lib.check(lib().rmt3d_profile_kernel(self._h, kernel, max_launches))

    def profile_read(self):
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        b = ctypes.c_double()
        _lib.check(lib().rmt3d_profile_read(self._h, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(b)))
        return ms.value, n.value, b.value

    def set_schedule(self, v_down, v_up, coarse_pts=-1):
        """Multigrid V(v_down, v_up) smoothing counts of both solvers and the
        largest level run by the one-block coarse sub-cycle (0: none,
        negative keeps it)."""
        _lib.check(lib().rmt3d_scene_set_schedule(self._h, v_down, v_up, coarse_pts))

    def set_mg_launch(self, cluster):
        """1: each multigrid solve as one thread-block-cluster launch; 0: one
        launch per phase in a graph loop."""
        _lib.check(lib().rmt3d_scene_set_mg_launch(self._h, int(cluster)))

    def set_smoother(self, mode):
        """Multigrid smoothing: 0 one launch per colour pass, 1 one launch per
        whole sweep on shared-memory tiles (the same bits)."""
        _lib.check(lib().rmt3d_scene_set_smoother(self._h, int(mode)))

    def set_coarse_cluster(self, pts):
        """Run the V-cycles' levels of at most `pts` points (below the finest)
        as one thread-block-cluster launch per cycle; 0: per-phase launches."""
        _lib.check(lib().rmt3d_scene_set_coarse_cluster(self._h, int(pts)))

    def set_block_shape(self, shape):
        """Block shape of the bulk stencil kernels by index (0: 32x4x2,
        1: 32x8x1, 2: 64x4x1, 3: 32x2x4, 4: 128x2x1; the same bits)."""
        _lib.check(lib().rmt3d_scene_set_block_shape(self._h, int(shape)))

    def snapshot(self, names, host_bufs):
        """Start copying the named fields to host buffers (objects with
        data_ptr(), e.g. pinned torch tensors of ncell doubles) without
        waiting; snapshot_wait() returns once they are in host memory."""
        which = (ctypes.c_int * len(names))(*[FIELD_INDEX[n] if isinstance(n, str) else int(n) for n in names])
        dst = (ctypes.c_void_p * len(names))(*[b.data_ptr() for b in host_bufs])
        _lib.check(lib().rmt3d_snapshot_fields(self._h, which, len(names), dst))

    def snapshot_wait(self):
        _lib.check(lib().rmt3d_snapshot_wait(self._h))

    def checksum(self):
        """Sums of u^2, v^2, w^2, p^2 over the interior cells."""
        out = (ctypes.c_double * 4)()
        _lib.check(lib().rmt3d_scene_checksum(self._h, out))
        return tuple(out)

    @property
    def device_bytes(self):
        """Device bytes the scene holds."""
        return int(self.scalar(12))

    def launches(self):
        c = ctypes.c_longlong()
        _lib.check(lib().rmt3d_launch_count(self._h, ctypes.byref(c)))
        return c.value

    def close(self):
        if getattr(self, "_h", None):
            lib().rmt3d_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Stepper:
    """Frame/step loop of the reference's stepper (Sim/stepper.hh:211-376):
    dt fit to frames, a restart's initial step and frame (chk_step,
    chk_num), stop_short counted from the initial step, and per frame the
    outputs of write_files and collect_macro_data (stepper.hh:378-474,
    578-610) that this path covers: tracer files with bit 1, slices of every
    out_flag type with bit 4, checkpoints every chkpt_freq frames with bit 8,
    macro.dat and centroid.dat with bit 32."""

    def __init__(self, desc, scene):
        self.dt, self.steps = stepper_dt(desc, desc.dt)
        run = desc.run
        self.init_step = run.chk_step
        self.init_frame = run.chk_num
        self.curr_tot_step = self.init_step
        self.frames = desc.frames
        self.total = (self.frames - 1) * self.steps
        self.stop_short = desc.stop_short + self.init_step if desc.stop_short > 0 else self.total + 1
        if self.frames - 1 > self.total:
            self.frames = self.total + 1
        self.dump_code = run.dump_code
        self.trace = run.ntracers > 0
        self.chkpt_freq = run.chkpt_freq
        self.dirname = run.dirname.decode()
        self.slices = []
        if self.dump_code & 4:
            self.slices = [(run.output_dim, run.output_ind, t, run.obj_body, run.data_fmt)
                           for t in range(len(OUTPUT_NAMES)) if (1 << t) & run.out_flag]
        scene.set_dt(self.dt)

    def write_files(self, scene, snum, fnum):
        if self.slices or (self.dump_code & 9):
            os.makedirs(self.dirname, exist_ok=True)
        if self.trace and (self.dump_code & 1):
            scene.write_tracers(os.path.join(self.dirname, "tr.%05d" % fnum), True)
            scene.write_tracers(os.path.join(self.dirname, "tr_st.%05d" % fnum), False)
        for dim, point, otype, obj_id, fmt in self.slices:
            scene.write_slice(otype, dim, point, obj_id, fmt,
                              os.path.join(self.dirname, "%s.%05d" % (OUTPUT_NAMES[otype], fnum)))
        if (self.dump_code & 8) and fnum % self.chkpt_freq == 0:
            scene.write_chk_pt(snum, fnum, os.path.join(self.dirname, "chk.%05d" % fnum))

    def collect_macro_data(self, scene, frame):
        """macro.dat and, with objects, centroid.dat, in the reference's
        layout (stepper.hh:378-474): a header when the file is new or at the
        initial step, then one record per frame (macro.dat's records carry
        no newline, as the reference writes them)."""
        if not self.dump_code & 32:
            return
        os.makedirs(self.dirname, exist_ok=True)
        fn = os.path.join(self.dirname, "macro.dat")
        if not os.path.exists(fn) or self.curr_tot_step == self.init_step:
            with open(fn, "w") as fh:
                fh.write("%10s %6s %6s %10s %6s %10s %6s %10s %10s %10s %10s %10s %10s %10s %10s %10s "
                         "%10s %10s %16s %16s %10s\n" % (
                             "#Time", "frame", "steps", "div_u_max", "rank", "div_u_min", "rank", "divu_L2",
                             "tot_mmt_x", "tot_mmt_y", "tot_mmt_z", "tot_energy", "kinetic", "elastic",
                             "potential", "power", "max_dev_detF", "dev_detF_L2", "sing. obj. cent.", "volume",
                             "change in u"))
        m = scene.macro()
        e = "%.15e"
        rec = ("%s %06d %06d %s %06d %s %06d " % (e % m.time, frame, self.curr_tot_step, e % m.div_u_max, 0,
                                                 e % m.div_u_min, 0))
        rec += e % m.div_u_l2 + " "
        rec += " ".join(e % v for v in (m.momentum[0], m.momentum[1], m.momentum[2], m.energy)) + " "
        rec += " ".join(e % v for v in (m.kinetic, m.elastic, m.potential, m.power)) + " "
        rec += " ".join(e % v for v in (m.max_dev_detF, m.dev_detF)) + " "
        with open(fn, "a") as fh:
            fh.write(rec)
        if m.n_obj > 0:
            fc = os.path.join(self.dirname, "centroid.dat")
            if not os.path.exists(fc) or self.curr_tot_step == self.init_step:
                with open(fc, "w") as fh:
                    fh.write("%10s %6s %6s %6s %6s %6s %6s %6s %6s->\n" % ("#Time", "frame", "steps", "x", "y", "z",
                                                                         "vx", "vy", "vz"))
            line = "%s %d %d " % (e % m.time, frame, self.curr_tot_step)
            for o in range(m.n_obj):
                line += " ".join(e % v for v in tuple(m.centroid[o]) + tuple(m.velocity[o])) + " "
            with open(fc, "a") as fh:
                fh.write(line + "\n")

    def run(self, scene):
        scene.set_dt(self.dt)
        self.write_files(scene, self.init_step, self.init_frame)
        self.collect_macro_data(scene, self.init_frame)
        err = 0
        frame = self.init_frame + 1
        while frame <= self.frames - 1 and self.curr_tot_step < self.stop_short:
            for _s in range(self.steps):
                if self.curr_tot_step >= self.stop_short:
                    break
                self.curr_tot_step += 1
                err = scene.step_forward(0)
                if err not in (NORMAL_EXIT, STEADY_SOLN_EXIT):
                    raise RMT3DError(err, "Stepper: Something went wrong, sorry.")
                if err == STEADY_SOLN_EXIT:
                    break
            self.write_files(scene, self.curr_tot_step, frame)
            self.collect_macro_data(scene, frame)
            if err == STEADY_SOLN_EXIT:
                break
            frame += 1
        return err


def run_sim(cfg_path, **overrides):
    """The run_sim driver sequence (Execs/run_sim.cc:64-141); returns the scene.
    A .cfg with chk_num > 0 (a checkpoint's recover.cfg) restarts from it."""
    desc = desc_from_cfg(cfg_path)
    for k, v in overrides.items():
        setattr(desc, k, v)
    scene = Scene(desc)
    init_err = scene.initialize()
    if scene.dt_reg < desc.dt:
        desc.dt = scene.dt_reg
    sim = Stepper(desc, scene)
    scene.init_iter(init_err)
    sim.run(scene)
    return scene


def footprint(desc):
    """Device bytes a scene with this descriptor allocates (admission control)."""
    return int(lib().rmt3d_scene_footprint(ctypes.byref(desc)))


class Batch:
    """Independent scenes stepped together, each on its own stream; a pool of
    host threads issues their steps so the kernels of many scenes overlap."""

    def __init__(self, descs, host_threads=0):
        L = lib()
        arr = (SceneDesc * len(descs))(*descs)
        h = ctypes.c_void_p()
        _lib.check(L.rmt3d_batch_create(arr, len(descs), host_threads, ctypes.byref(h)))
        self._h = h
        self.n = len(descs)

    def prepare(self):
        _lib.check(lib().rmt3d_batch_prepare(self._h))

    def step(self, nsteps=1):
        st = (ctypes.c_int * self.n)()
        _lib.check(lib().rmt3d_batch_step(self._h, nsteps, st))
        return list(st)

    def scene_handle(self, i):
        h = ctypes.c_void_p()
        _lib.check(lib().rmt3d_batch_scene(self._h, i, ctypes.byref(h)))
        return h

    def checksum(self, i):
        out = (ctypes.c_double * 4)()
        _lib.check(lib().rmt3d_scene_checksum(self.scene_handle(i), out))
        return tuple(out)

    def field(self, i, name):
        h = self.scene_handle(i)
        dims = (ctypes.c_int * 6)()
        _lib.check(lib().rmt3d_get_dims(h, dims))
        n = dims[0] * dims[1] * dims[2]
        out = np.empty(n, dtype=np.float64)
        idx = FIELD_INDEX[name] if isinstance(name, str) else int(name)
        _lib.check(lib().rmt3d_get_field(h, idx, out.ctypes.data_as(ctypes.c_void_p)))
        return out.reshape(dims[2], dims[1], dims[0])

    def autotune(self, probe_steps=3):
        """Per kind of scene: {cells: (v_down, v_up, cluster, smoother,
        coarse cluster points, block shape)} chosen by timing candidates
        (smoother 0: colour passes, 1: tiled sweeps; block shape as in
        Scene.set_block_shape)."""
        buf = (ctypes.c_int * (7 * self.n))()
        n = ctypes.c_int()
        _lib.check(lib().rmt3d_batch_autotune(self._h, probe_steps, buf, self.n, ctypes.byref(n)))
        return {buf[7 * i]: tuple(buf[7 * i + 1:7 * i + 7]) for i in range(min(n.value, self.n))}

    def set_smoother(self, mode):
        """The multigrid smoother of every scene (Scene.set_smoother)."""
        _lib.check(lib().rmt3d_batch_set_smoother(self._h, int(mode)))

    def close(self):
        if getattr(self, "_h", None):
            lib().rmt3d_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve(requests, hbm_budget, max_slots, grouped=False):
    """Run a request stream [(arrival_s, steps, desc), ...] through the serving
    loop (grouped: requests of one kind stepped as one group graph); returns
    (per-request result dicts, summary dict)."""
    L = lib()
    n = len(requests)
    reqs = (_lib.Request * n)()
    for i, (arr, steps, desc) in enumerate(requests):
        reqs[i].arrival_s = arr
        reqs[i].steps = steps
        reqs[i].desc = desc
    res = (_lib.RequestResult * n)()
    summ = _lib.ServeSummary()
    fn = L.rmt3d_serve_grouped if grouped else L.rmt3d_serve
    _lib.check(fn(reqs, n, hbm_budget, max_slots, res, ctypes.byref(summ)))

    def as_dict(st):
        out = {}
        for name, _t in st._fields_:
            v = getattr(st, name)
            out[name] = tuple(v) if hasattr(v, "__len__") else v
        return out

    return [as_dict(r) for r in res], as_dict(summ)
