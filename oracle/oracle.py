"""Python access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

* ``Oracle``: ctypes binding of the plain-C restatement (oracle/_build/liboracle.so).
* ``run_reference``: runs the unmodified reference build (oracle/_ref/torch_ref)
  in a fresh process per case and reads its ``TRGS`` state dump.

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline leg of bench.py
import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
LIB_PM_PATH = os.path.join(HERE, "_build", "liboracle_pm.so")
REF_BIN = os.path.join(HERE, "_ref", "torch_ref")
# the reference source tree: $TORCH_REFERENCE, default /root/reference
REF_TREE = os.environ.get("TORCH_REFERENCE", "/root/reference")


class OrcParams(C.Structure):
    _fields_ = [
        ("dscale", C.c_double), ("pscale", C.c_double), ("tscale", C.c_double),
        ("spatial_order", C.c_int), ("temporal_order", C.c_int),
        ("tmax", C.c_double),
        ("radiation_on", C.c_int), ("cooling_on", C.c_int),
        ("nd", C.c_int), ("ncells", C.c_int * 3),
        ("side_length", C.c_double),
        ("geometry", C.c_int), ("left_bc", C.c_int * 3), ("right_bc", C.c_int * 3),
        ("gamma", C.c_double), ("dfloor", C.c_double), ("tfloor", C.c_double),
        ("riemann", C.c_int), ("limiter", C.c_int),
        ("K1", C.c_double), ("K2", C.c_double), ("K3", C.c_double), ("K4", C.c_double),
        ("photoion_xsec", C.c_double), ("alphaB", C.c_double), ("tau0", C.c_double),
        ("minX", C.c_double), ("THI", C.c_double), ("THII", C.c_double), ("mass_frac_h", C.c_double),
        ("rt_scheme", C.c_int), ("collisions_on", C.c_int), ("coupling", C.c_int),
        ("heating_amp", C.c_double), ("thermo_hii_switch", C.c_double),
        ("thermo_subcycling", C.c_int), ("min_temp_initial_state", C.c_int),
        ("star_on", C.c_int), ("star_pos", C.c_int * 3), ("face_snap", C.c_int * 3),
        ("photon_energy", C.c_double), ("photon_rate", C.c_double), ("mass_loss_rate", C.c_double),
        ("wind_velocity", C.c_double), ("wind_temperature", C.c_double),
        ("wind_cell_radius", C.c_int),
    ]


def build(quiet: bool = True, portable_math: bool = False) -> str:
    """Compiles the C restatement (make -C oracle) if it is missing or stale."""
    src = os.path.join(HERE, "torch_oracle.c")
    path = LIB_PM_PATH if portable_math else LIB_PATH
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE], check=True,
                       stdout=subprocess.DEVNULL if quiet else None)
    return path


def build_reference(quiet: bool = True) -> Optional[str]:
    """Builds oracle/_ref/torch_ref from the reference sources when they are present."""
    if os.path.exists(REF_BIN):
        return REF_BIN
    if not os.path.isdir(os.path.join(REF_TREE, "src")):
        return None
    subprocess.run(["make", "-C", os.path.join(HERE, "ref"), f"REF={REF_TREE}", "-j8"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
    return REF_BIN if os.path.exists(REF_BIN) else None


_libs = {}


def _load(portable_math: bool = False):
    if portable_math not in _libs:
        _lib = C.CDLL(build(portable_math=portable_math))
        _libs[portable_math] = _lib
        _lib.orc_create.restype = C.c_void_p
        _lib.orc_create.argtypes = [C.POINTER(OrcParams)] + [C.c_void_p] * 7 + [C.c_char_p, C.c_int]
        _lib.orc_full_step.restype = C.c_int
        _lib.orc_full_step.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_double)]
        _lib.orc_get_state.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        _lib.orc_time.restype = C.c_double
        _lib.orc_time.argtypes = [C.c_void_p]
        _lib.orc_dt_max.restype = C.c_double
        _lib.orc_dt_max.argtypes = [C.c_void_p]
        _lib.orc_ncells.restype = C.c_long
        _lib.orc_ncells.argtypes = [C.c_void_p]
        _lib.orc_last_error.restype = C.c_char_p
        _lib.orc_last_error.argtypes = [C.c_void_p]
        _lib.orc_destroy.argtypes = [C.c_void_p]
        _lib.orc_causal_order.restype = C.c_long
        _lib.orc_causal_order.argtypes = [C.c_void_p, C.c_void_p, C.c_long]
        _lib.orc_cell_volumes.restype = C.c_long
        _lib.orc_cell_volumes.argtypes = [C.c_void_p, C.c_void_p, C.c_long]
        _lib.orc_set_libm_noise.argtypes = [C.c_double]
    return _libs[portable_math]


def set_libm_noise(fraction: float) -> None:
    """Test hook of the host-libm oracle: from now on a fixed, input-determined
    fraction of its exp/log/log10/pow results is moved by one ulp (0: off).
    Process-wide: it applies to every host-libm Oracle of this process."""
    _load(False).orc_set_libm_noise(float(fraction))


def params_struct(tp, side_length: Optional[float] = None, ncells=None) -> OrcParams:
    """Fills the raw-parameter struct from a torch_b200.config.TorchParameters."""
    from torch_b200.config import CONDITION, GEOMETRY, enum_value
    p = OrcParams()
    p.dscale, p.pscale, p.tscale = tp.dscale, tp.pscale, tp.tscale
    p.spatial_order, p.temporal_order = tp.spatialOrder, tp.temporalOrder
    p.tmax = tp.tmax
    p.radiation_on, p.cooling_on = int(tp.radiation_on), int(tp.cooling_on)
    nc = ncells if ncells is not None else tp.ncells
    p.nd = 1 if nc[1] == 1 else (2 if nc[2] == 1 else 3)
    for i in range(3):
        p.ncells[i] = nc[i]
        p.left_bc[i] = enum_value(CONDITION, tp.leftBC[i])
        p.right_bc[i] = enum_value(CONDITION, tp.rightBC[i])
        p.star_pos[i] = tp.star_position[i]
        p.face_snap[i] = int(tp.faceSnap[i])
    p.side_length = tp.sideLength if side_length is None else side_length
    p.geometry = enum_value(GEOMETRY, tp.geometry)
    p.gamma, p.dfloor, p.tfloor = tp.heatCapacityRatio, tp.dfloor, tp.tfloor
    p.riemann, p.limiter = tp.riemann_id(), tp.limiter_id()
    p.K1, p.K2, p.K3, p.K4 = tp.K1, tp.K2, tp.K3, tp.K4
    p.photoion_xsec, p.alphaB, p.tau0 = tp.photoIonCrossSection, tp.alphaB, tp.tau0
    p.minX, p.THI, p.THII, p.mass_frac_h = tp.minX, tp.THI, tp.THII, tp.massFractionH
    p.rt_scheme, p.collisions_on, p.coupling = tp.scheme_id(), int(tp.collisions_on), tp.coupling_id()
    p.heating_amp, p.thermo_hii_switch = tp.heatingAmplification, tp.thermoHII_Switch
    p.thermo_subcycling, p.min_temp_initial_state = int(tp.thermoSubcycling), int(tp.minTempInitialState)
    p.star_on = int(tp.star_on)
    p.photon_energy, p.photon_rate = tp.photonEnergy, tp.photonRate
    p.mass_loss_rate, p.wind_velocity = tp.massLossRate, tp.windVelocity
    p.wind_temperature, p.wind_cell_radius = tp.windTemperature, tp.windCellRadius
    return p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class State:
    U: np.ndarray
    Q: np.ndarray
    R: np.ndarray
    T: np.ndarray
    Tmin: np.ndarray
    time: float
    dts: np.ndarray


class Oracle:
    """The C restatement, driven like Torch::run (one context per run).

    portable_math=False: host libm, bit-exact with the reference build.
    portable_math=True: the exp/log/log10/pow of torch_b200/csrc/trg_math.h
    (correctly rounded, IEEE operations only) that the FP64 GPU kernels use,
    i.e. the GPU's bit-exact CPU twin."""

    def __init__(self, tp, ic, portable_math: bool = False):
        lib = _load(portable_math)
        self.N = int(np.prod(ic.ncells))
        p = params_struct(tp, side_length=ic.side_length, ncells=ic.ncells)
        err = C.create_string_buffer(512)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                (ic.den, ic.pre, ic.hii, ic.vel[0], ic.vel[1], ic.vel[2])]
        grav = getattr(ic, "grav", None)
        garr = None if grav is None else np.ascontiguousarray(grav, dtype=np.float64)
        self._keep = arrs + [garr]
        self.ctx = lib.orc_create(C.byref(p), *[_ptr(a) for a in arrs], _ptr(garr), err, 512)
        if not self.ctx:
            raise RuntimeError("oracle: " + err.value.decode())
        self.lib = lib
        self.dts = []

    def full_step(self, dt_next: Optional[float] = None) -> float:
        dt = C.c_double(0)
        if dt_next is None:
            dt_next = self.lib.orc_dt_max(self.ctx)
        rc = self.lib.orc_full_step(self.ctx, dt_next, C.byref(dt))
        if rc:
            raise RuntimeError(f"oracle step failed ({rc}): " + self.lib.orc_last_error(self.ctx).decode())
        self.dts.append(dt.value)
        return dt.value

    def state(self) -> State:
        N = self.N
        U = np.zeros((7, N)); Q = np.zeros((7, N)); R = np.zeros((6, N)); T = np.zeros((4, N)); Tm = np.zeros(N)
        self.lib.orc_get_state(self.ctx, _ptr(U), _ptr(Q), _ptr(R), _ptr(T), _ptr(Tm))
        return State(U, Q, R, T, Tm, self.lib.orc_time(self.ctx), np.array(self.dts))

    def causal_order(self) -> np.ndarray:
        out = np.zeros(self.N, dtype=np.int32)
        n = self.lib.orc_causal_order(self.ctx, _ptr(out), self.N)
        return out[:n]

    def cell_volumes(self) -> np.ndarray:
        """Cell volumes in code units (Grid::computeCellVolume, Grid.cpp:876-905)."""
        out = np.zeros(self.N)
        self.lib.orc_cell_volumes(self.ctx, _ptr(out), self.N)
        return out

    def close(self):
        if self.ctx:
            self.lib.orc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def exact_sum_of_products(a, b) -> float:
    """sum_i a_i b_i of two FP64 arrays, computed exactly (rational
    arithmetic) and rounded once to the nearest double: the checker of the
    library's global conservation sums."""
    from fractions import Fraction
    total = Fraction(0)
    for x, y in zip(np.asarray(a, dtype=np.float64).tolist(), np.asarray(b, dtype=np.float64).tolist()):
        total += Fraction(x) * Fraction(y)
    return float(total)


def conservation_sums(U, vol):
    """Exact global (mass, energy) = (sum rho V, sum E V) of a conserved state
    U [7][N] with cell volumes vol [N]."""
    return exact_sum_of_products(U[0], vol), exact_sum_of_products(U[1], vol)


def read_trgs(path: str) -> State:
    """Reads the TRGS dump written by oracle/ref/ref_driver.cpp."""
    raw = np.fromfile(path, dtype=np.uint8)
    hdr = np.frombuffer(raw[:32].tobytes(), dtype=np.int32)
    if raw[:4].tobytes() != b"TRGS":
        raise ValueError(f"{path}: not a TRGS dump")
    nx, ny, nz, nd, nsteps = (int(v) for v in hdr[2:7])
    t, dx = np.frombuffer(raw[32:48].tobytes(), dtype=np.float64)
    N = nx * ny * nz
    a = np.frombuffer(raw[48:].tobytes(), dtype=np.float64)
    o = 0
    out = []
    for n in (7, 7, 6, 4, 1):
        out.append(a[o:o + n * N].reshape(n, N).copy())
        o += n * N
    dts = a[o:o + nsteps].copy()
    return State(out[0], out[1], out[2], out[3], out[4][0], float(t), dts)


def run_reference(params_path: str, ic_path: Optional[str], steps: int, workdir: str,
                  setup_path: Optional[str] = None, timeout: float = 600, print2d: Optional[str] = None,
                  setup_dump: Optional[str] = None) -> State:
    """Runs the reference binary on a case in a fresh process and returns its final state
    (with `print2d`, the reference also writes its checkpoint files of that state there)."""
    binp = build_reference()
    if binp is None:
        raise FileNotFoundError("reference build unavailable (oracle/_ref/torch_ref)")
    out = os.path.join(workdir, f"ref_{steps}.bin")
    cmd = [binp, f"--params={params_path}", f"--steps={steps}", f"--out={out}"]
    if ic_path:
        cmd.append(f"--ic={ic_path}")
    if setup_path:
        cmd.append(f"--setup={setup_path}")
    if print2d:
        cmd.append(f"--print2d={print2d}")
    if setup_dump:
        cmd.append(f"--setup-dump={setup_dump}")
    r = subprocess.run(cmd, cwd=workdir, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed ({r.returncode}): {r.stderr[-2000:]}")
    return read_trgs(out)
