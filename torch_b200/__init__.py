"""torch_b200: B200-native TORCH operator-split timestep behind a C ABI.

The compute path is ``libtorch_b200.so`` (hand-written sm_100a CUDA kernels,
built in-tree by ``torch_b200/csrc/Makefile``).  This module binds its C ABI
(``include/torch_b200.h``) with ctypes and mirrors the reference's driver
interface (``Torch::initialise`` / ``Torch::fullStep`` / ``Torch::run``,
src/Torch/Torch.cpp) so that Python callers and the tests drive it like the
reference.  There is no CPU fallback: if the library is missing or no GPU is
present, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import config
from .config import CONDITION, GEOMETRY, TorchParameters, enum_value

__all__ = ["Torch", "TrgError", "library_path", "load_library", "TorchParameters", "config",
           "initial_conditions_from_lua", "setup_positions"]

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_NAME = "libtorch_b200.so"

PRECISION_FP64 = 0
PRECISION_FP32 = 1

COMP_HYDRO, COMP_RAD, COMP_THERMO, COMP_FLUID = 0, 1, 2, 3
PHASE_PRE, PHASE_DT, PHASE_INTEGRATE, PHASE_SOURCES, PHASE_Q_FROM_U, PHASE_ADVANCE = 0, 1, 2, 3, 4, 5

ERROR_NAMES = {1: "TRG_ERR_ARG", 2: "TRG_ERR_CUDA", 3: "TRG_ERR_NAN", 4: "TRG_ERR_PICARD",
               5: "TRG_ERR_DT", 6: "TRG_ERR_FLUX", 7: "TRG_ERR_OOM", 8: "TRG_ERR_TC", 9: "TRG_ERR_SUBCYCLE"}


class TrgError(RuntimeError):
    """A failing torch_b200 call (the reference throws std::runtime_error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


class TrgParams(C.Structure):
    """ctypes mirror of ``trg_params`` (include/torch_b200.h)."""
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
        ("precision", C.c_int),
        ("device", C.c_int),
    ]


def library_path() -> str:
    return os.path.join(HERE, _LIB_NAME)


_lib = None

# (name, restype, argtypes) for every entry point of include/torch_b200.h
# the x-slab exchange hook of trg_slab_exchange: int fn(void* user, int what, void* stream)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p)
EXCHANGE_HALO, EXCHANGE_DT, EXCHANGE_SWEEP_IN, EXCHANGE_SWEEP_OUT = 0, 1, 2, 3

_SIGNATURES = [
    ("trg_create", C.c_int, [C.POINTER(TrgParams)] + [C.c_void_p] * 7 + [C.POINTER(C.c_void_p)]),
    ("trg_setup_positions", C.c_int, [C.POINTER(TrgParams)] + [C.c_void_p] * 4),
    ("trg_full_step", C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_double)]),
    ("trg_run_steps", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    ("trg_component", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.POINTER(C.c_double)]),
    ("trg_get_state", C.c_int, [C.c_void_p] + [C.c_void_p] * 5),
    ("trg_set_conserved", C.c_int, [C.c_void_p, C.c_void_p]),
    ("trg_synchronize", C.c_int, [C.c_void_p]),
    ("trg_time", C.c_double, [C.c_void_p]),
    ("trg_dt_max", C.c_double, [C.c_void_p]),
    ("trg_ncells", C.c_long, [C.c_void_p]),
    ("trg_kernel_launches", C.c_longlong, [C.c_void_p]),
    ("trg_last_error", C.c_char_p, [C.c_void_p]),
    ("trg_destroy", None, [C.c_void_p]),
    ("trg_enqueue_steps", C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    ("trg_stream", C.c_void_p, [C.c_void_p]),
    ("trg_profile_enable", C.c_int, [C.c_void_p, C.c_int]),
    ("trg_profile_read", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    ("trg_stats_enable", C.c_int, [C.c_void_p, C.c_int]),
    ("trg_autotune", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    ("trg_checkpoint_bytes", C.c_longlong, [C.c_void_p]),
    ("trg_heating_enable", C.c_int, [C.c_void_p, C.c_int]),
    ("trg_fp32_contrast", C.c_int, [C.c_void_p, C.c_double]),
    ("trg_thermo_queue", C.c_int, [C.c_void_p, C.c_int]),
    ("trg_fp32_tma", C.c_int, [C.c_void_p, C.c_int]),
    ("trg_heating", C.c_int, [C.c_void_p, C.c_void_p]),
    ("trg_checkpoint_save", C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong]),
    ("trg_checkpoint_load", C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong]),
    ("trg_mlp_create", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    ("trg_mlp_get_params", C.c_int, [C.c_void_p, C.c_void_p]),
    ("trg_mlp_set_params", C.c_int, [C.c_void_p, C.c_void_p]),
    ("trg_mlp_forward", C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_void_p]),
    ("trg_mlp_gradient", C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_double)]),
    ("trg_mlp_train", C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_float, C.c_uint,
                                C.c_void_p, C.c_void_p]),
    ("trg_mlp_last_error", C.c_char_p, [C.c_void_p]),
    ("trg_mlp_destroy", None, [C.c_void_p]),
    ("trg_learned_start", C.c_int, [C.c_void_p, C.c_void_p]),
    ("trg_batch_create", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    ("trg_batch_run_steps", C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    ("trg_batch_enqueue_steps", C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    ("trg_batch_step_graphs", C.c_int, [C.c_void_p, C.c_int]),
    ("trg_batch_learned_start", C.c_int, [C.c_void_p, C.c_void_p]),
    ("trg_batch_set_conserved", C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    ("trg_batch_get_conserved", C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    ("trg_batch_synchronize", C.c_int, [C.c_void_p]),
    ("trg_batch_stream", C.c_void_p, [C.c_void_p]),
    ("trg_batch_kernel_launches", C.c_longlong, [C.c_void_p]),
    ("trg_batch_cells", C.c_longlong, [C.c_void_p]),
    ("trg_batch_profile_enable", C.c_int, [C.c_void_p, C.c_int]),
    ("trg_batch_profile_read", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    ("trg_batch_last_error", C.c_char_p, [C.c_void_p]),
    ("trg_batch_destroy", None, [C.c_void_p]),
    ("trg_harvest", C.c_int, [C.c_void_p, C.c_long]),
    ("trg_harvest_read", C.c_long, [C.c_void_p, C.c_void_p, C.c_long]),
    ("trg_stats", C.c_int, [C.c_void_p, C.POINTER(C.c_ulonglong), C.c_int]),
    ("trg_conservation_sums", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("trg_conservation_enable", C.c_int, [C.c_void_p, C.c_int]),
    ("trg_conservation_history", C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.POINTER(C.c_longlong)]),
    ("trg_hydro_step_fp32_noalloc", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.POINTER(C.c_double), C.c_void_p]),
    ("trg_create_slab", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p] + [C.c_void_p] * 7
     + [C.POINTER(C.c_void_p)]),
    ("trg_slab_exchange", C.c_int, [C.c_void_p, EXCHANGE_FN, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("trg_slab_halo_bytes", C.c_longlong, [C.c_void_p]),
    ("trg_slab_partitions", C.c_int, [C.c_void_p]),
    ("trg_slab_sweep_exchange", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("trg_fp32_tile", C.c_int, [C.c_void_p, C.c_int]),
    ("trg_slab_sweep_bytes", C.c_longlong, [C.c_void_p]),
    ("trg_slab_star_side", C.c_int, [C.c_void_p]),
    ("trg_f32_scales", C.c_int, [C.c_void_p] + [C.c_void_p] * 6 + [C.c_void_p]),
]


def load_library():
    """Loads libtorch_b200.so from the package directory (raises if absent)."""
    global _lib
    if _lib is None:
        path = library_path()
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing: build it with `make -C torch_b200/csrc` "
                                    "(there is no CPU fallback)")
        lib = C.CDLL(path)
        for name, res, args in _SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


NSTATS = 24
PICARD_BINS = ("1", "2", "3-4", "5-8", "9-16", "17-64", "65-1024", ">1024")


def make_params(tp: TorchParameters, side_length: float, ncells, precision: int = PRECISION_FP64,
                device: int = 0) -> TrgParams:
    p = TrgParams()
    p.dscale, p.pscale, p.tscale = tp.dscale, tp.pscale, tp.tscale
    p.spatial_order, p.temporal_order = tp.spatialOrder, tp.temporalOrder
    p.tmax = tp.tmax
    p.radiation_on, p.cooling_on = int(tp.radiation_on), int(tp.cooling_on)
    p.nd = 1 if ncells[1] == 1 else (2 if ncells[2] == 1 else 3)
    for i in range(3):
        p.ncells[i] = int(ncells[i])
        p.left_bc[i] = enum_value(CONDITION, tp.leftBC[i])
        p.right_bc[i] = enum_value(CONDITION, tp.rightBC[i])
        p.star_pos[i] = tp.star_position[i]
        p.face_snap[i] = int(tp.faceSnap[i])
    p.side_length = side_length
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
    p.precision = precision
    p.device = device
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


MLP_NPARAMS = 4755
MLP_NTRAIN = 4739
MLP_IN, MLP_HID, MLP_OUT = 5, 64, 3


def mlp_init_params(seed: int = 0) -> np.ndarray:
    """He-initialised parameter vector (biases zero, identity normalisation)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(MLP_NPARAMS, dtype=np.float32)
    o = 0
    for fan_in, fan_out in ((MLP_IN, MLP_HID), (MLP_HID, MLP_HID), (MLP_HID, MLP_OUT)):
        p[o:o + fan_in * fan_out] = rng.normal(0.0, np.sqrt(2.0 / fan_in), fan_in * fan_out)
        o += fan_in * fan_out + fan_out
    p[MLP_NTRAIN + 5:MLP_NTRAIN + 10] = 1.0   # input scale
    p[MLP_NTRAIN + 13:MLP_NTRAIN + 16] = 1.0  # output scale
    return p


class Mlp:
    """The learned starting iterate's network on one GPU (trg_mlp_*)."""

    def __init__(self, params=None, device: int = 0, seed: int = 0):
        self.lib = load_library()
        p = np.ascontiguousarray(mlp_init_params(seed) if params is None else params, dtype=np.float32)
        if p.size != MLP_NPARAMS:
            raise ValueError(f"expected {MLP_NPARAMS} parameters")
        h = C.c_void_p()
        rc = self.lib.trg_mlp_create(p.ctypes.data_as(C.c_void_p), int(device), C.byref(h))
        if rc != 0:
            raise TrgError(rc, "trg_mlp_create failed")
        self.handle = h.value

    def _check(self, rc):
        if rc != 0:
            raise TrgError(rc, self.lib.trg_mlp_last_error(self.handle).decode())

    def params(self) -> np.ndarray:
        p = np.zeros(MLP_NPARAMS, dtype=np.float32)
        self._check(self.lib.trg_mlp_get_params(self.handle, p.ctypes.data_as(C.c_void_p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self.lib.trg_mlp_set_params(self.handle, p.ctypes.data_as(C.c_void_p)))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, MLP_IN)
        y = np.zeros((x.shape[0], MLP_OUT), dtype=np.float32)
        self._check(self.lib.trg_mlp_forward(self.handle, x.ctypes.data_as(C.c_void_p), x.shape[0],
                                             y.ctypes.data_as(C.c_void_p)))
        return y

    def gradient(self, records, out_weight=(1.0, 1.0, 1.0)):
        r = np.ascontiguousarray(records, dtype=np.float32).reshape(-1, 8)
        w = np.ascontiguousarray(out_weight, dtype=np.float32)
        g = np.zeros(MLP_NTRAIN, dtype=np.float32)
        loss = C.c_double(0)
        self._check(self.lib.trg_mlp_gradient(self.handle, r.ctypes.data_as(C.c_void_p), r.shape[0],
                                              w.ctypes.data_as(C.c_void_p), g.ctypes.data_as(C.c_void_p),
                                              C.byref(loss)))
        return g, loss.value

    def train(self, records, epochs=10, batch=4096, lr=1e-3, seed=0, out_weight=(1.0, 0.25, 0.1)):
        r = np.ascontiguousarray(records, dtype=np.float32).reshape(-1, 8)
        w = np.ascontiguousarray(out_weight, dtype=np.float32)
        hist = np.zeros(max(epochs, 1), dtype=np.float32)
        self._check(self.lib.trg_mlp_train(self.handle, r.ctypes.data_as(C.c_void_p), r.shape[0], int(epochs),
                                           int(batch), float(lr), int(seed), w.ctypes.data_as(C.c_void_p),
                                           hist.ctypes.data_as(C.c_void_p)))
        return hist[:epochs]

    def close(self):
        if getattr(self, "handle", None):
            self.lib.trg_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def setup_positions(tp: TorchParameters):
    """(x, y, z, star) in cgs as Torch::setUpLua passes them to the Lua setup
    function (src/Torch/Torch.cpp:196-228), computed by the library's host
    code (no GPU needed)."""
    lib = load_library()
    ncells = tuple(tp.ncells)
    p = make_params(tp, tp.sideLength, ncells)
    N = int(np.prod(ncells))
    x, y, z, star = np.zeros(N), np.zeros(N), np.zeros(N), np.zeros(3)
    rc = lib.trg_setup_positions(C.byref(p), _ptr(x), _ptr(y), _ptr(z), _ptr(star))
    if rc != 0:
        raise TrgError(rc, "trg_setup_positions: invalid grid parameters")
    return x, y, z, star


def initial_conditions_from_lua(tp: TorchParameters, setup) -> "config.InitialConditions":
    """Initial conditions from a Lua setup script (a path or a
    ``lua_setup.LuaScript``): the script's ``initialise(x, y, z, xs, ys, zs)``
    evaluated for every cell of the grid ``tp`` describes, as
    Torch::setUpLua does (src/Torch/Torch.cpp:196-228), gravity included."""
    from . import lua_setup
    script = setup if isinstance(setup, lua_setup.LuaScript) else lua_setup.LuaScript.from_file(setup)
    x, y, z, star = setup_positions(tp)
    v = lua_setup.evaluate_setup(script, x, y, z, star)
    ic = config.make_initial_conditions(tuple(tp.ncells), tp.sideLength / tp.ncells[0], v["den"], v["pre"],
                                        v["hii"], v["vel"])
    ic.side_length = tp.sideLength
    ic.grav = v["grav"]
    return ic


class Torch:
    """One run on one GPU: ``Torch::initialise`` then ``full_step`` calls.

    ``ic`` is a ``config.InitialConditions`` (primitives in cgs, as the
    reference's DataReader or Lua setup provides them).
    """

    def __init__(self, tp: TorchParameters, ic, precision: int = PRECISION_FP64, device: int = 0, slab=None):
        """slab = (x0, nx, f32_scale or None): this context holds global x from
        x0 to x0 + nx - 1 of the grid `ic` describes (trg_create_slab); the
        step then needs an exchange hook (torch_b200.slabs)."""
        self.lib = load_library()
        p = make_params(tp, ic.side_length, ic.ncells, precision, device)
        fields = [ic.den, ic.pre, ic.hii, ic.vel[0], ic.vel[1], ic.vel[2]]
        grav = getattr(ic, "grav", None)
        if slab is not None:
            x0, nx = int(slab[0]), int(slab[1])
            shape = (int(ic.ncells[2]), int(ic.ncells[1]), int(ic.ncells[0]))
            fields = [np.asarray(a, dtype=np.float64).reshape(shape)[:, :, x0:x0 + nx].ravel() for a in fields]
            if grav is not None:
                grav = np.asarray(grav, dtype=np.float64).reshape((3,) + shape)[:, :, :, x0:x0 + nx].reshape(3, -1)
            self.N = nx * shape[0] * shape[1]
        else:
            self.N = int(np.prod(ic.ncells))
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in fields]
        garr = None if grav is None else np.ascontiguousarray(grav, dtype=np.float64)
        ctx = C.c_void_p()
        if slab is not None:
            sc = None if slab[2] is None else np.ascontiguousarray(slab[2], dtype=np.float64)
            rc = self.lib.trg_create_slab(C.byref(p), x0, nx, _ptr(sc), *[_ptr(a) for a in arrs], _ptr(garr),
                                          C.byref(ctx))
        else:
            rc = self.lib.trg_create(C.byref(p), *[_ptr(a) for a in arrs], _ptr(garr), C.byref(ctx))
        self.ctx = ctx.value
        if rc != 0:
            msg = self.lib.trg_last_error(self.ctx).decode() if self.ctx else "trg_create failed"
            self.close()
            raise TrgError(rc, msg)
        self.dts = []

    def _check(self, rc):
        if rc != 0:
            raise TrgError(rc, self.lib.trg_last_error(self.ctx).decode())

    @property
    def dt_max(self) -> float:
        return self.lib.trg_dt_max(self.ctx)

    def full_step(self, dt_next_checkpoint: Optional[float] = None) -> float:
        """Torch::fullStep (src/Torch/Torch.cpp:389-418); returns dt."""
        if dt_next_checkpoint is None:
            dt_next_checkpoint = self.dt_max
        dt = C.c_double(0)
        self._check(self.lib.trg_full_step(self.ctx, dt_next_checkpoint, C.byref(dt)))
        self.dts.append(dt.value)
        return dt.value

    def run_steps(self, nsteps: int, dt_next_checkpoint: Optional[float] = None) -> np.ndarray:
        """nsteps full steps enqueued back to back; returns their dt values."""
        if dt_next_checkpoint is None:
            dt_next_checkpoint = self.dt_max
        out = np.zeros(max(nsteps, 1))
        self._check(self.lib.trg_run_steps(self.ctx, nsteps, dt_next_checkpoint, _ptr(out)))
        self.dts.extend(out[:nsteps].tolist())
        return out[:nsteps]

    def enqueue_steps(self, nsteps: int, dt_next_checkpoint: Optional[float] = None):
        """Enqueues nsteps full steps and returns at once (see synchronize())."""
        if dt_next_checkpoint is None:
            dt_next_checkpoint = self.dt_max
        self._check(self.lib.trg_enqueue_steps(self.ctx, nsteps, dt_next_checkpoint))

    def stream_handle(self) -> int:
        return int(self.lib.trg_stream(self.ctx) or 0)

    def profile(self, on: bool):
        self._check(self.lib.trg_profile_enable(self.ctx, int(on)))

    def profile_read(self, name: str):
        ms = C.c_double(0)
        n = C.c_longlong(0)
        self._check(self.lib.trg_profile_read(self.ctx, name.encode(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def learned_start(self, mlp):
        """Start the front cells' ionisation solve from `mlp` (an Mlp), or plain with None."""
        self._check(self.lib.trg_learned_start(self.ctx, mlp.handle if mlp is not None else None))

    def harvest(self, capacity: int):
        """Record up to `capacity` front-cell training records from the plain solve (0 stops)."""
        self._check(self.lib.trg_harvest(self.ctx, int(capacity)))

    def harvest_read(self, max_records: int = 1 << 26, count_only: bool = False):
        """(records [k x 8] float32, total recorded) of the current harvest;
        with count_only, just the number recorded so far."""
        n = int(self.lib.trg_harvest_read(self.ctx, None, 0))
        if n < 0:
            raise TrgError(-n, "trg_harvest_read failed")
        if count_only:
            return n
        k = min(n, int(max_records))
        out = np.zeros((k, 8), dtype=np.float32)
        if k:
            got = int(self.lib.trg_harvest_read(self.ctx, out.ctypes.data_as(C.c_void_p), k))
            if got < 0:
                raise TrgError(-got, "trg_harvest_read failed")
        return out, n

    def fp32_contrast(self, contrast: float):
        """Pressure ratio above which the FP32 form updates a hydro cell in FP64 (0: off)."""
        self._check(self.lib.trg_fp32_contrast(self.ctx, float(contrast)))

    def fp32_tma(self, on: bool):
        """FP32 hydro pass on the FP64 state: stage planes by TMA where possible (default on)."""
        self._check(self.lib.trg_fp32_tma(self.ctx, int(on)))

    def thermo_queue(self, min_subcycles: int):
        """Cells with at least this many thermal sub-cycles run through the
        work queue (0: all in place)."""
        self._check(self.lib.trg_thermo_queue(self.ctx, int(min_subcycles)))

    def conservation_sums(self):
        """Global FP64 (mass, energy) = (sum rho V, sum E V) of the current state."""
        m, e = C.c_double(0), C.c_double(0)
        self._check(self.lib.trg_conservation_sums(self.ctx, C.byref(m), C.byref(e)))
        return m.value, e.value

    def conservation_enable(self, on: bool = True):
        """Record the conservation sums of the state every step starts from."""
        self._check(self.lib.trg_conservation_enable(self.ctx, int(on)))

    def conservation_history(self) -> np.ndarray:
        """[n, 2] recorded (mass, energy); row k is the state after k steps."""
        n = C.c_longlong(0)
        self._check(self.lib.trg_conservation_history(self.ctx, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 2))
        self._check(self.lib.trg_conservation_history(self.ctx, _ptr(out), n.value, C.byref(n)))
        return out[:n.value]

    def heating_enable(self, on: bool = True):
        """Keep the heating/cooling terms during the step (for heating())."""
        self._check(self.lib.trg_heating_enable(self.ctx, int(on)))

    def heating(self) -> np.ndarray:
        """Thermodynamics::fillHeatingArrays: the 11 terms [11, N] in code units."""
        H = np.zeros((11, self.N), dtype=np.float64)
        self._check(self.lib.trg_heating(self.ctx, H.ctypes.data_as(C.c_void_p)))
        return H

    def checkpoint(self) -> bytes:
        """The whole step state as bytes (trg_checkpoint_save)."""
        n = int(self.lib.trg_checkpoint_bytes(self.ctx))
        buf = (C.c_char * n)()
        self._check(self.lib.trg_checkpoint_save(self.ctx, buf, n))
        return bytes(buf)

    def restore(self, blob: bytes):
        """Continues from a checkpoint of a run with the same parameters and grid."""
        self._check(self.lib.trg_checkpoint_load(self.ctx, blob, len(blob)))

    def autotune(self):
        """Tile depth of the FP32 hydro kernel chosen by timing; (zchunk, ms per launch)."""
        z = C.c_int(0)
        ms = C.c_double(0)
        self._check(self.lib.trg_autotune(self.ctx, C.byref(z), C.byref(ms)))
        return z.value, ms.value

    def set_tile(self, zchunk: int) -> int:
        """Sets the FP32 hydro kernel's tile depth (z planes per CTA); returns the depth in effect."""
        return int(self.lib.trg_fp32_tile(self.ctx, int(zchunk)))

    def stats_enable(self, on: bool):
        self._check(self.lib.trg_stats_enable(self.ctx, int(on)))

    def stats(self, reset: bool = False) -> dict:
        """Solver counters (TRG_STAT_* of the C header) as a dict."""
        buf = (C.c_ulonglong * NSTATS)()
        self._check(self.lib.trg_stats(self.ctx, buf, int(reset)))
        v = list(buf)
        return {"picard_cells": v[0], "picard_iters": v[1], "picard_max": v[2],
                "picard_hist": dict(zip(PICARD_BINS, v[3:11])),
                "learned_cells": v[11], "learned_accepted": v[12], "learned_iters": v[13],
                "thermo_cells": v[14], "thermo_subcycles": v[15], "thermo_max": v[16], "sweeps": v[17],
                "front_cells": v[18], "front_iters": v[19], "fp64_cells": v[20]}

    def component(self, comp: int, phase: int, dt: float = 0.0) -> float:
        out = C.c_double(0)
        self._check(self.lib.trg_component(self.ctx, comp, phase, dt, C.byref(out)))
        return out.value

    def state(self) -> State:
        N = self.N
        U = np.zeros((7, N)); Q = np.zeros((7, N)); R = np.zeros((6, N)); T = np.zeros((4, N)); Tm = np.zeros(N)
        self._check(self.lib.trg_get_state(self.ctx, _ptr(U), _ptr(Q), _ptr(R), _ptr(T), _ptr(Tm)))
        return State(U, Q, R, T, Tm, self.lib.trg_time(self.ctx), np.array(self.dts))

    def set_conserved(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64)
        self._check(self.lib.trg_set_conserved(self.ctx, _ptr(U)))

    def kernel_launches(self) -> int:
        return int(self.lib.trg_kernel_launches(self.ctx))

    def synchronize(self):
        self._check(self.lib.trg_synchronize(self.ctx))

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.trg_destroy(self.ctx)
            self.ctx = None

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
    """Independent grids advanced together, one launch per stage (trg_batch_*).

    `grids` are fresh FP64 ``Torch`` runs with the same physics flags; they
    are stepped only through the batch while it exists, and their states are
    read with their own ``state()`` after ``synchronize()``.
    """

    def __init__(self, grids):
        self.lib = load_library()
        self.grids = list(grids)
        arr = (C.c_void_p * len(self.grids))(*[g.ctx for g in self.grids])
        h = C.c_void_p()
        rc = self.lib.trg_batch_create(arr, len(self.grids), C.byref(h))
        if rc != 0:
            msgs = [g.lib.trg_last_error(g.ctx).decode() for g in self.grids]
            raise TrgError(rc, next((m for m in msgs if m), "trg_batch_create failed"))
        self.handle = h.value
        self.cells = int(self.lib.trg_batch_cells(self.handle))

    def _check(self, rc):
        if rc != 0:
            raise TrgError(rc, self.lib.trg_batch_last_error(self.handle).decode())

    def run_steps(self, nsteps: int, dt_next_checkpoint: float):
        self._check(self.lib.trg_batch_run_steps(self.handle, int(nsteps), float(dt_next_checkpoint)))

    def enqueue_steps(self, nsteps: int, dt_next_checkpoint: float):
        self._check(self.lib.trg_batch_enqueue_steps(self.handle, int(nsteps), float(dt_next_checkpoint)))

    def set_conserved(self, g: int, U_ptr: int):
        """Copy grid g's conserved state in from host memory at U_ptr (pinned
        for an asynchronous copy), on the batch's stream."""
        self._check(self.lib.trg_batch_set_conserved(self.handle, int(g), C.c_void_p(U_ptr)))

    def get_conserved(self, g: int, U_ptr: int):
        """Copy grid g's conserved state out to host memory at U_ptr, on the batch's stream."""
        self._check(self.lib.trg_batch_get_conserved(self.handle, int(g), C.c_void_p(U_ptr)))

    def step_graphs(self, on: bool):
        """One captured CUDA graph per timestep (on by default)."""
        self._check(self.lib.trg_batch_step_graphs(self.handle, int(on)))

    def learned_start(self, mlp):
        """The learned starting iterate for every grid of the batch (an ``Mlp``
        on the batch's device), or the plain solve again (None)."""
        self._check(self.lib.trg_batch_learned_start(self.handle, mlp.handle if mlp is not None else None))

    def synchronize(self):
        self._check(self.lib.trg_batch_synchronize(self.handle))

    def stream_handle(self) -> int:
        return int(self.lib.trg_batch_stream(self.handle) or 0)

    def kernel_launches(self) -> int:
        return int(self.lib.trg_batch_kernel_launches(self.handle))

    def profile(self, on: bool):
        self._check(self.lib.trg_batch_profile_enable(self.handle, int(on)))

    def profile_read(self, name: str):
        ms = C.c_double(0)
        n = C.c_longlong(0)
        self._check(self.lib.trg_batch_profile_read(self.handle, name.encode(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def close(self):
        if getattr(self, "handle", None):
            self.lib.trg_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
