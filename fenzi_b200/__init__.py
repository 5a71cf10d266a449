"""fenzi_b200 — B200-native (sm_100a) FEN ZI molecular-dynamics step.

Python host mirror of the reference's driver-facing functions, over the C ABI of
``libfenzi_b200.so`` (declared in include/fenzi_b200.h).  Method names follow the
reference (src/fenzi.cu main() call sequence):

    sys = FenZi.ReadInput("fenzi.in")   # ReadInput            src/prmread.cu:491
    sys.LoadSystem()                    # LoadCoord, ReadPsf_CHARMM, ReadPrm_CHARMM,
                                        # build_constraints, GenExcl_minimal_new
    sys.InitMem(device=0)               # InitMem + InitDeviceConstants
    sys.InitVelocity()                  # InitVelocity         src/init.cu:19
    sys.ComputeAccelGPU()               # ComputeAccelGPU      src/mdcuda.cu:557
    sys.SingleStep(n)                   # SingleStep x n       src/dynamics.cu:623
    e = sys.EvalProps()                 # EvalProps            src/evalprops.cu:17

Errors raise FenZiError carrying the library's status code and message (the
reference prints and calls exit()).  There is no CPU fallback: if the CUDA library
is missing the import of the compute path fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfenzi_b200.so")

E_FIELDS = ["bond", "angle", "ureyb", "dihed", "impr", "vdw", "elec", "pme", "ewexcl", "ewself",
            "potential", "kinetic", "temperature"]

STATUS = {0: "OK", 1: "IO", 2: "PARSE", 3: "CUDA", 4: "CAPACITY", 5: "SHAKE", 6: "ARG", 7: "STATE",
          8: "NOMEM", 9: "TIMEOUT"}


class FenZiError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{STATUS.get(code, code)}] {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [
        ("coordinates", C.c_char * 512), ("structure", C.c_char * 512), ("parameters", C.c_char * 512),
        ("topology", C.c_char * 512), ("outputname", C.c_char * 512), ("outputtrajectory", C.c_char * 512),
        ("restartfilename", C.c_char * 512),
        ("temperature", C.c_double), ("thermostat", C.c_double), ("temp_reset_every", C.c_int),
        ("minimize_steps", C.c_int), ("conjgradfac", C.c_double), ("steepdesfac", C.c_double),
        ("conjgradrate", C.c_double), ("steepdesrate", C.c_double),
        ("start_step", C.c_int), ("timestep_ps", C.c_double), ("dyna_steps", C.c_int),
        ("kappa", C.c_double), ("inbfrq", C.c_int), ("output_every", C.c_int), ("checkpoint_every", C.c_int),
        ("traj_every", C.c_int), ("cuton", C.c_double), ("cutoff", C.c_double), ("pairlistdist", C.c_double),
        ("gpublocksize", C.c_int), ("box", C.c_double * 3), ("pme_grid", C.c_int * 3),
        ("pmass", C.c_double), ("pref", C.c_double), ("shake", C.c_int), ("shake_tol", C.c_double),
        ("hfac", C.c_double), ("printlevel", C.c_int), ("printtostdout", C.c_int), ("keepcheckpoints", C.c_int),
        ("checkpointformat", C.c_char), ("seed", C.c_longlong), ("unknown_keywords", C.c_int),
        ("consharm", C.c_int), ("consharm_seg", (C.c_char * 64) * 2), ("consharm_dist", C.c_double * 3),
        ("consharm_fc", C.c_double), ("consfix_nseg", C.c_int), ("consfix_seg", (C.c_char * 64) * 8),
    ]


class Energies(C.Structure):
    _fields_ = [(k, C.c_double) for k in E_FIELDS] + [
        ("virial", C.c_double * 3), ("pressure_atm", C.c_double), ("step", C.c_longlong),
        ("box", C.c_double * 3), ("volume", C.c_double), ("conserved", C.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k in E_FIELDS}
        d.update(virial=list(self.virial), pressure_atm=self.pressure_atm, step=self.step, box=list(self.box),
                 volume=self.volume, conserved=self.conserved)
        return d


class JobInfo(C.Structure):
    _fields_ = [("job", C.c_int), ("state", C.c_int), ("status", C.c_int), ("natom", C.c_int),
                ("nsteps", C.c_longlong), ("steps_done", C.c_longlong), ("submit_s", C.c_double),
                ("start_s", C.c_double), ("end_s", C.c_double), ("device_bytes", C.c_double), ("final", Energies)]


class Info(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("natom", "ntypes", "nbond", "nangle", "nureyb", "ndihedral", "nimproper",
                                       "nconstraint", "ncluster", "nexcl_pairs", "n14_pairs", "ndihedral_terms")] + [
        ("pme_grid", C.c_int * 3), ("box", C.c_double * 3)]


# exported symbols of include/fenzi_b200.h
EXPORTS = ["fz_last_error", "fz_version", "fz_read_input", "fz_load_system", "fz_get_info", "fz_get_array",
           "fz_free", "fz_upload", "fz_reassign_velocities", "fz_compute_forces", "fz_compute_forces_terms", "fz_step", "fz_eval_props",
           "fz_get_positions", "fz_set_positions", "fz_get_velocities", "fz_set_velocities", "fz_get_forces",
           "fz_get_forces_fixed", "fz_set_state_f32", "fz_get_state_f32", "fz_get_counters", "fz_get_launch_shapes", "fz_sync",
           "fz_stream", "fz_set_stage_timing", "fz_get_stage_times", "fz_measure_fp32_peak",
           "fz_pme_reciprocal_static", "fz_batch_create", "fz_batch_add", "fz_batch_step", "fz_batch_free",
           "fz_set_barostat", "fz_get_virial", "fz_batch_remove", "fz_batch_size", "fz_server_create",
           "fz_server_submit", "fz_server_info", "fz_server_wait", "fz_server_positions", "fz_server_stats",
           "fz_server_free", "fz_server_estimate_bytes", "fz_checkpoint_save", "fz_checkpoint_load",
           "fz_dcd_open", "fz_dcd_write", "fz_dcd_close", "fz_minimize"]

STAGES = ["neighbour", "nonbonded", "bonded", "pme", "integrate"]

TERM_NONBONDED, TERM_BONDED, TERM_PME, TERM_ALL = 1, 2, 4, 7
# parts of TERM_BONDED, selectable one by one
TERM_BONDS, TERM_ANGLES, TERM_UREYB, TERM_DIHEDRALS, TERM_IMPROPERS, TERM_PAIRS14, TERM_EXCLUSIONS = (
    8, 16, 32, 64, 128, 256, 512)

_lib = None


def lib():
    """Loads libfenzi_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m fenzi_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        sig = {
            "fz_last_error": ([C.c_char_p, C.c_size_t], C.c_int),
            "fz_version": ([], C.c_char_p),
            "fz_read_input": ([C.c_char_p, C.POINTER(Config)], C.c_int),
            "fz_load_system": ([C.POINTER(Config), C.POINTER(vp)], C.c_int),
            "fz_get_info": ([vp, C.POINTER(Info)], C.c_int),
            "fz_get_array": ([vp, C.c_char_p, vp, C.c_size_t], C.c_int),
            "fz_free": ([vp], C.c_int),
            "fz_upload": ([vp, C.c_int, vp], C.c_int),
            "fz_reassign_velocities": ([vp, C.c_double, C.c_uint64, C.c_uint32], C.c_int),
            "fz_compute_forces": ([vp, C.c_int], C.c_int),
            "fz_compute_forces_terms": ([vp, C.c_int, C.c_int], C.c_int),
            "fz_step": ([vp, C.c_int], C.c_int),
            "fz_eval_props": ([vp, C.POINTER(Energies)], C.c_int),
            "fz_get_positions": ([vp, dp], C.c_int),
            "fz_set_positions": ([vp, dp], C.c_int),
            "fz_get_velocities": ([vp, dp], C.c_int),
            "fz_set_velocities": ([vp, dp], C.c_int),
            "fz_get_forces": ([vp, dp], C.c_int),
            "fz_get_forces_fixed": ([vp, C.POINTER(C.c_longlong)], C.c_int),
            "fz_set_state_f32": ([vp, vp, vp], C.c_int),
            "fz_get_state_f32": ([vp, vp, vp], C.c_int),
            "fz_get_counters": ([vp, C.POINTER(C.c_longlong)], C.c_int),
            "fz_get_launch_shapes": ([vp, C.POINTER(C.c_int)], C.c_int),
            "fz_sync": ([vp], C.c_int),
            "fz_set_stage_timing": ([vp, C.c_int], C.c_int),
            "fz_get_stage_times": ([vp, dp], C.c_int),
            "fz_measure_fp32_peak": ([C.c_int, dp], C.c_int),
            "fz_batch_create": ([C.POINTER(vp)], C.c_int),
            "fz_batch_add": ([vp, vp], C.c_int),
            "fz_batch_step": ([vp, C.c_int], C.c_int),
            "fz_batch_free": ([vp], C.c_int),
            "fz_pme_reciprocal_static": ([C.c_int, vp, vp, C.c_int, dp, C.POINTER(C.c_int), C.c_double, vp, dp],
                                         C.c_int),
            "fz_stream": ([vp], vp),
            "fz_set_barostat": ([vp, C.c_int, C.c_double, C.c_double], C.c_int),
            "fz_get_virial": ([vp, dp], C.c_int),
            "fz_batch_remove": ([vp, vp], C.c_int),
            "fz_batch_size": ([vp, C.POINTER(C.c_int)], C.c_int),
            "fz_server_create": ([C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
            "fz_server_submit": ([vp, vp, C.c_longlong, C.POINTER(C.c_int)], C.c_int),
            "fz_server_info": ([vp, C.c_int, C.POINTER(JobInfo)], C.c_int),
            "fz_server_wait": ([vp, C.c_int, C.POINTER(JobInfo)], C.c_int),
            "fz_server_positions": ([vp, C.c_int, dp], C.c_int),
            "fz_server_stats": ([vp, dp], C.c_int),
            "fz_server_free": ([vp], C.c_int),
            "fz_server_estimate_bytes": ([vp, dp], C.c_int),
            "fz_checkpoint_save": ([vp, C.c_char_p, C.c_int], C.c_int),
            "fz_checkpoint_load": ([vp, C.c_char_p, C.c_int], C.c_int),
            "fz_dcd_open": ([vp, C.c_char_p, C.c_int, C.POINTER(vp)], C.c_int),
            "fz_dcd_write": ([vp], C.c_int),
            "fz_dcd_close": ([vp], C.c_int),
            "fz_minimize": ([vp, C.c_int, C.POINTER(C.c_int), dp], C.c_int),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def last_error():
    buf = C.create_string_buffer(2048)
    lib().fz_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def _check(code):
    if code != 0:
        raise FenZiError(code, last_error())


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class FenZi:
    """One system (one fz_system handle)."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.h = C.c_void_p()
        self.n = 0

    # ---- input (host only)
    @classmethod
    def ReadInput(cls, path: str) -> "FenZi":
        cfg = Config()
        _check(lib().fz_read_input(path.encode(), C.byref(cfg)))
        return cls(cfg)

    def LoadSystem(self):
        _check(lib().fz_load_system(C.byref(self.cfg), C.byref(self.h)))
        self.n = self.info().natom
        return self

    def info(self) -> Info:
        i = Info()
        _check(lib().fz_get_info(self.h, C.byref(i)))
        return i

    def array(self, name: str, count: int, dtype) -> np.ndarray:
        out = np.zeros(count, dtype=dtype)
        _check(lib().fz_get_array(self.h, name.encode(), out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def topology(self) -> dict:
        """Parsed topology (for inspection and tests)."""
        i = self.info()
        nt = i.ntypes
        d = dict(n=i.natom, ntypes=nt)
        d["pos"] = self.array("pos", 3 * i.natom, np.float64).reshape(-1, 3)
        d["q"] = self.array("q", i.natom, np.float64)
        d["mass"] = self.array("mass", i.natom, np.float64)
        d["type"] = self.array("type", i.natom, np.int32)
        for k in ("eps4", "sig2", "eps4_14", "sig2_14"):
            d[k] = self.array(k, nt * nt, np.float64).reshape(nt, nt)
        d["bond"] = self.array("bond", 2 * i.nbond, np.int32).reshape(-1, 2)
        d["bond_k"], d["bond_r0"] = self.array("bond_k", i.nbond, np.float64), self.array("bond_r0", i.nbond, np.float64)
        d["angle"] = self.array("angle", 3 * i.nangle, np.int32).reshape(-1, 3)
        d["angle_k"] = self.array("angle_k", i.nangle, np.float64)
        d["angle_t0"] = self.array("angle_t0", i.nangle, np.float64)
        d["ub"] = self.array("ureyb", 2 * i.nureyb, np.int32).reshape(-1, 2)
        d["ub_k"], d["ub_r0"] = self.array("ureyb_k", i.nureyb, np.float64), self.array("ureyb_r0", i.nureyb, np.float64)
        nd = i.ndihedral_terms
        d["dihe"] = self.array("dihe", 4 * nd, np.int32).reshape(-1, 4)
        d["dihe_k"], d["dihe_n"] = self.array("dihe_k", nd, np.float64), self.array("dihe_n", nd, np.int32)
        d["dihe_d"] = self.array("dihe_d", nd, np.float64)
        d["impr"] = self.array("impr", 4 * i.nimproper, np.int32).reshape(-1, 4)
        d["impr_k"] = self.array("impr_k", i.nimproper, np.float64)
        d["impr_p0"] = self.array("impr_p0", i.nimproper, np.float64)
        d["cons"] = self.array("cons", 2 * i.nconstraint, np.int32).reshape(-1, 2)
        d["cons_d"] = self.array("cons_d", i.nconstraint, np.float64)
        d["excl"] = self.array("excl", 2 * i.nexcl_pairs, np.int32).reshape(-1, 2)
        d["p14"] = self.array("p14", 2 * i.n14_pairs, np.int32).reshape(-1, 2)
        c = self.cfg
        d.update(box=np.array(list(c.box)), rc=c.cutoff, ron=c.cuton, beta=c.kappa, K=np.array(list(c.pme_grid)))
        return d

    # ---- device
    def InitMem(self, device: int = 0, stream=None):
        _check(lib().fz_upload(self.h, int(device), stream))
        return self

    def InitVelocity(self, T: float | None = None, seed: int | None = None, counter: int = 0):
        T = self.cfg.temperature if T is None else T
        seed = self.cfg.seed if seed is None else seed
        _check(lib().fz_reassign_velocities(self.h, float(T), int(seed) & (2 ** 64 - 1), int(counter)))

    def ComputeAccelGPU(self, energies: bool = False, terms: int = 7):
        """Forces (and energies) at the current positions; terms: TERM_* bit mask."""
        if terms == TERM_ALL:
            _check(lib().fz_compute_forces(self.h, 1 if energies else 0))
        else:
            _check(lib().fz_compute_forces_terms(self.h, int(terms), 1 if energies else 0))

    def SingleStep(self, nsteps: int = 1):
        _check(lib().fz_step(self.h, int(nsteps)))

    def EvalProps(self) -> dict:
        e = Energies()
        _check(lib().fz_eval_props(self.h, C.byref(e)))
        return e.as_dict()

    def Minimize(self, nsteps: int | None = None):
        """MinimizeStep loop (CG then SD); returns (moves made, final potential energy)."""
        k, e = C.c_int(), C.c_double()
        n = self.cfg.minimize_steps if nsteps is None else nsteps
        _check(lib().fz_minimize(self.h, int(n), C.byref(k), C.byref(e)))
        return k.value, e.value

    def SaveCheckpoint(self, path: str, fmt: str | None = None):
        """Restart file in the reference's layout: fmt 'a' (ascii), 'b' (binary) or None
        (the input's checkpointformat)."""
        _check(lib().fz_checkpoint_save(self.h, path.encode(), ord(fmt) if fmt else 0))

    def LoadCheckpoint(self, path: str, fmt: str | None = None):
        _check(lib().fz_checkpoint_load(self.h, path.encode(), ord(fmt) if fmt else 0))

    def set_barostat(self, enable: bool = True, pref_atm: float | None = None, pmass: float | None = None):
        """Andersen constant-pressure dynamics (the reference's PCONSTANT build) for the
        following SingleStep calls; defaults are the input file's pref / pmass."""
        pr = self.cfg.pref if pref_atm is None else pref_atm
        pm = self.cfg.pmass if pmass is None else pmass
        _check(lib().fz_set_barostat(self.h, 1 if enable else 0, float(pr), float(pm)))

    def positions(self):
        out = np.zeros((self.n, 3))
        _check(lib().fz_get_positions(self.h, _dp(out)))
        return out

    def set_positions(self, pos):
        p = np.ascontiguousarray(pos, np.float64)
        _check(lib().fz_set_positions(self.h, _dp(p)))

    def velocities(self):
        out = np.zeros((self.n, 3))
        _check(lib().fz_get_velocities(self.h, _dp(out)))
        return out

    def set_velocities(self, vel):
        v = np.ascontiguousarray(vel, np.float64)
        _check(lib().fz_set_velocities(self.h, _dp(v)))

    def forces(self):
        out = np.zeros((self.n, 3))
        _check(lib().fz_get_forces(self.h, _dp(out)))
        return out

    def forces_fixed(self):
        out = np.zeros(3 * self.n, np.int64)
        _check(lib().fz_get_forces_fixed(self.h, out.ctypes.data_as(C.POINTER(C.c_longlong))))
        return out

    def set_state_f32(self, pos, vel):
        _check(lib().fz_set_state_f32(self.h, pos.ctypes.data_as(C.c_void_p) if pos is not None else None,
                                      vel.ctypes.data_as(C.c_void_p) if vel is not None else None))

    def get_state_f32(self, pos, vel):
        _check(lib().fz_get_state_f32(self.h, pos.ctypes.data_as(C.c_void_p) if pos is not None else None,
                                      vel.ctypes.data_as(C.c_void_p) if vel is not None else None))

    def counters(self):
        out = (C.c_longlong * 4)()
        _check(lib().fz_get_counters(self.h, out))
        return dict(launches=out[0], rebuilds=out[1], pair_slots=out[2], prunes=out[3])

    def launch_shapes(self):
        """Launch shapes in use: pair tiles per work item, pair-kernel CTAs per SM, PME
        brick edge per dimension, gather kernel, and whether the autotuner picked them."""
        out = (C.c_int * 7)()
        _check(lib().fz_get_launch_shapes(self.h, out))
        return dict(chunk_tiles=out[0], nb_ctas_per_sm=out[1], pme_brick=[out[2], out[3], out[4]],
                    gather={0: "auto", 1: "brick", 2: "atom", 3: "atom-spread"}[out[5]], autotuned=bool(out[6]))

    def stage_timing(self, enable=True):
        _check(lib().fz_set_stage_timing(self.h, 1 if enable else 0))

    def stage_times(self):
        """Mean milliseconds per step of each stage over the steps timed so far."""
        out = np.zeros(6)
        _check(lib().fz_get_stage_times(self.h, _dp(out)))
        n = max(1.0, out[5])
        return {k: out[i] / n for i, k in enumerate(STAGES)} | {"steps": int(out[5])}

    def sync(self):
        _check(lib().fz_sync(self.h))

    def virial(self):
        """Virial diagonal of the last ComputeAccelGPU(..., energies=True)-style call."""
        out = np.zeros(3)
        _check(lib().fz_get_virial(self.h, _dp(out)))
        return out

    def stream(self):
        return lib().fz_stream(self.h)

    def close(self):
        if self.h:
            lib().fz_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fp32_peak_tflops(device: int = 0) -> float:
    out = C.c_double()
    _check(lib().fz_measure_fp32_peak(int(device), C.byref(out)))
    return out.value


class Batch:
    """Independent systems advanced together, one CUDA-graph launch per MD step."""

    def __init__(self, systems=()):
        self.h = C.c_void_p()
        _check(lib().fz_batch_create(C.byref(self.h)))
        self.systems = []
        for s in systems:
            self.add(s)

    def add(self, s: FenZi):
        _check(lib().fz_batch_add(self.h, s.h))
        self.systems.append(s)

    def remove(self, s: FenZi):
        _check(lib().fz_batch_remove(self.h, s.h))
        self.systems.remove(s)

    def step(self, nsteps=1):
        _check(lib().fz_batch_step(self.h, int(nsteps)))

    def close(self):
        if self.h:
            lib().fz_batch_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving loop (fz_server_*): submitted jobs are admitted by an HBM budget, stay
    resident and advance together in the batch graph; each job's latency is measured
    from submission to completion on the server's clock."""

    STATES = ("queued", "running", "done", "failed")

    def __init__(self, device=0, hbm_budget_bytes=150e9, chunk_steps=100, max_running=64):
        self.h = C.c_void_p()
        _check(lib().fz_server_create(int(device), float(hbm_budget_bytes), int(chunk_steps), int(max_running),
                                      C.byref(self.h)))
        self.natom = {}

    @staticmethod
    def estimate_bytes(s: FenZi) -> float:
        """Admission estimate of a loaded system's device memory."""
        out = C.c_double()
        _check(lib().fz_server_estimate_bytes(s.h, C.byref(out)))
        return out.value

    def submit(self, s: FenZi, nsteps: int) -> int:
        """Hands a loaded (not uploaded) system to the server, which owns it from now on."""
        jid = C.c_int()
        _check(lib().fz_server_submit(self.h, s.h, int(nsteps), C.byref(jid)))
        self.natom[jid.value] = s.n
        s.h = C.c_void_p()
        return jid.value

    @staticmethod
    def _as_dict(j: JobInfo) -> dict:
        return dict(job=j.job, state=Server.STATES[j.state], status=j.status, natom=j.natom, nsteps=j.nsteps,
                    steps_done=j.steps_done, submit_s=j.submit_s, start_s=j.start_s, end_s=j.end_s,
                    latency_s=j.end_s - j.submit_s if j.end_s >= 0 else None, device_bytes=j.device_bytes,
                    final=j.final.as_dict())

    def info(self, job: int) -> dict:
        j = JobInfo()
        _check(lib().fz_server_info(self.h, int(job), C.byref(j)))
        return self._as_dict(j)

    def wait(self, job: int) -> dict:
        j = JobInfo()
        _check(lib().fz_server_wait(self.h, int(job), C.byref(j)))
        return self._as_dict(j)

    def positions(self, job: int):
        out = np.zeros((self.natom[job], 3))
        _check(lib().fz_server_positions(self.h, int(job), _dp(out)))
        return out

    def stats(self) -> dict:
        out = np.zeros(4)
        _check(lib().fz_server_stats(self.h, _dp(out)))
        return dict(peak_running=int(out[0]), atom_steps=int(out[1]), bytes_in_use=out[2], finished=int(out[3]))

    def close(self):
        if self.h:
            _check(lib().fz_server_free(self.h))
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Trajectory:
    """CHARMM DCD trajectory of one system (fz_dcd_*): write() appends the current frame."""

    def __init__(self, system: FenZi, path: str, every: int = 1):
        self.h = C.c_void_p()
        _check(lib().fz_dcd_open(system.h, path.encode(), int(every), C.byref(self.h)))

    def write(self):
        _check(lib().fz_dcd_write(self.h))

    def close(self):
        if self.h:
            _check(lib().fz_dcd_close(self.h))
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def pme_reciprocal_static(device, pos4_ptr, n, box, K, beta, facc_ptr, stream=None, energy=True):
    """PME reciprocal forces with no device allocation (fz_pme_reciprocal_static):
    pos4_ptr / facc_ptr are caller-owned device pointers (float4[n], int64[3n])."""
    b = (C.c_double * 3)(*[float(x) for x in box])
    k = (C.c_int * 3)(*[int(x) for x in K])
    e = C.c_double()
    _check(lib().fz_pme_reciprocal_static(int(device), stream, C.c_void_p(pos4_ptr), int(n), b, k, float(beta),
                                          C.c_void_p(facc_ptr), C.byref(e) if energy else None))
    return e.value if energy else None


def load(in_path: str, device: int | None = None) -> FenZi:
    """ReadInput + LoadSystem (+ InitMem when device is given)."""
    s = FenZi.ReadInput(in_path).LoadSystem()
    if device is not None:
        s.InitMem(device)
    return s
