"""Test infrastructure: ctypes binding of the CPU restatement of the reference
sheet step (oracle/sheet_oracle.cpp). Only the parity tests, the smoke check and
the CPU-baseline leg of bench.py load it; the product never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_silt.so")

_f = ctypes.c_float
_i = ctypes.c_int
_p = ctypes.c_void_p


def _structs(real):
    """The interface's structures with `real` for every float field (the
    FP64 build's interface carries doubles)."""

    class CoreCfg(ctypes.Structure):
        _fields_ = [("res", _i), ("cell", real), ("fine_res", _i), ("fine_cell", real),
                    ("layout", _i), ("tire_r", real), ("soften", _i), ("inner_par", _i),
                    ("center_x", real), ("center_z", real), ("threads", _i)]

    class Tire(ctypes.Structure):
        _fields_ = [("x", real), ("z", real), ("forward_x", real), ("forward_z", real),
                    ("radius", real), ("width", real), ("speed", real), ("slip", real)]

    class Spray(ctypes.Structure):
        _fields_ = [("x", real), ("y", real), ("z", real), ("vx", real), ("vy", real), ("vz", real),
                    ("volume", real), ("kind", _i)]

    return CoreCfg, Tire, Spray


CoreCfg, Tire, Spray = _structs(_f)
CoreCfg64, Tire64, Spray64 = _structs(ctypes.c_double)


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


NATIVE_PATH = os.path.join(HERE, "_native", "liboracle_silt.so")
NATIVE_FLAGS = "-O3 -march=native -ffp-contract=off"


def use_native_build(timeout=300):
    """Loads the -O3 -march=native build (compiled here on first use) in
    place of the portable one; must come before the first call. Returns the
    flags of the build in use."""
    global LIB_PATH
    if _lib is not None:
        return NATIVE_FLAGS if LIB_PATH == NATIVE_PATH else "-O2 -ffp-contract=off"
    try:
        subprocess.run(["make", "-s", "-C", HERE, "native"], check=True, timeout=timeout,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        LIB_PATH = NATIVE_PATH
        return NATIVE_FLAGS
    except (subprocess.SubprocessError, OSError):
        return "-O2 -ffp-contract=off"


_lib = None
_lib64 = None
LIB64_PATH = os.path.join(HERE, "liboracle_silt_f64.so")


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = _bind(ctypes.CDLL(LIB_PATH), _f, CoreCfg, Tire)
    return _lib


def lib64():
    """The FP64 restatement (same source, built with -DORACLE_F64)."""
    global _lib64
    if _lib64 is None:
        if not os.path.exists(LIB64_PATH):
            build()
        _lib64 = _bind(ctypes.CDLL(LIB64_PATH), ctypes.c_double, CoreCfg64, Tire64)
    return _lib64


_lib_rn = None
LIB_RN_PATH = os.path.join(HERE, "liboracle_silt_rn.so")


def lib_rn():
    """The step with the device's elementary functions (-DORACLE_ELEM_RN)."""
    global _lib_rn
    if _lib_rn is None:
        if not os.path.exists(LIB_RN_PATH):
            build()
        _lib_rn = _bind(ctypes.CDLL(LIB_RN_PATH), _f, CoreCfg, Tire)
    return _lib_rn


def _bind(L, _f, CoreCfg, Tire):
    if True:
        L.oracle_scratch_new.restype = _p
        L.oracle_scratch_free.argtypes = [_p]
        L.oracle_step_sheet.argtypes = [_p, _p, _p, _p, _p, _p, _i, _f, _f, _f, _f, _i, _f, _i, _i, _p]
        L.oracle_transport_open.argtypes = [_p, _p, _p, _i, _f, _f, _i, _i, _i, _i, _i, _p, _f, _i, _p, _p]
        L.oracle_sheet_work_boxes.argtypes = [_p, _i, _f, _i, _i, _p, _i]
        L.oracle_awake_work_boxes.argtypes = [_p, _p, _p, _p, _i, _f, _f, _p, _i]
        L.oracle_dynamic_viscosity.argtypes = [_i, _f]
        L.oracle_dynamic_viscosity.restype = _f
        L.oracle_sheet_mobility_for.argtypes = [_f]
        L.oracle_sheet_mobility_for.restype = _f
        L.oracle_sheet_damp.argtypes = [_f]
        L.oracle_sheet_damp.restype = _f
        L.oracle_soften_border.argtypes = [_p, _p, _i]
        L.oracle_rut_heal.argtypes = [_i, _f, _p]
        L.oracle_core_new.argtypes = [ctypes.POINTER(CoreCfg)]
        L.oracle_core_new.restype = _p
        L.oracle_core_free.argtypes = [_p]
        L.oracle_core_map_water_bed.argtypes = [_p, _p, _p]
        L.oracle_core_map_water_bed.restype = _f
        L.oracle_core_map_grain.argtypes = [_p, _p]
        L.oracle_core_map_water_velocity.argtypes = [_p, _p, _p]
        L.oracle_core_pour.argtypes = [_p, _f, _f, _f, _f, _f, _i, _i, _f]
        L.oracle_core_pour.restype = _f
        L.oracle_core_lay_slurry_mask.argtypes = [_p, _p, _i, _f]
        L.oracle_core_lay_slurry_mask.restype = _f
        L.oracle_core_read_substrate.argtypes = [_p, _p, _p, _p]
        L.oracle_core_push_tire.argtypes = [_p, ctypes.POINTER(Tire)]
        L.oracle_core_step.argtypes = [_p, _f, _p, _i]
        L.oracle_core_step.restype = _i
        L.oracle_core_ledger.argtypes = [_p, _p, _p]
        L.oracle_core_get.argtypes = [_p, _i, _p]
        L.oracle_core_set.argtypes = [_p, _i, _p]
        L.oracle_core_get_grain.argtypes = [_p, _p]
        L.oracle_core_publish.argtypes = [_p, _p, _p]
        L.oracle_core_set_fine_pace.argtypes = [_p, _i]
        L.oracle_core_set_turbidity.argtypes = [_p, _i]
        L.oracle_core_set_reach_turbidity.argtypes = [_p, _f]
        L.oracle_core_tracer_books.argtypes = [_p, _p, _p]
        L.oracle_core_set_fine_sub_cap.argtypes = [_p, _f]
        L.oracle_core_set_near_field.argtypes = [_p, _i]
        L.oracle_core_set_open_water.argtypes = [_p, _i, _f, _f, _f]
        L.oracle_core_set_surface_diffusion.argtypes = [_p, _f]
        L.oracle_core_recenter.argtypes = [_p, _f, _f]
        L.oracle_core_set_river_reach.argtypes = [_p, _i, _i, _i, _f, _f, _i, _f, _f, _f]
        L.oracle_core_reach_bank.argtypes = [_p]
        L.oracle_core_reach_bank.restype = _f
        L.oracle_core_set_wave_maker.argtypes = [_p, _i, _f, _f, _f, _f, _f, _f, _f, _f, _f]
        L.oracle_core_origin.argtypes = [_p, _p]
        L.oracle_core_parked_count.argtypes = [_p]
        L.oracle_core_parked_count.restype = _i
        L.oracle_core_near_tiles.argtypes = [_p]
        L.oracle_core_near_tiles.restype = _i
        L.oracle_core_spray_m3.argtypes = [_p]
        L.oracle_core_spray_m3.restype = _f
        L.oracle_core_non_finite.argtypes = [_p]
        L.oracle_core_non_finite.restype = ctypes.c_uint32
        L.oracle_core_sample.argtypes = [_p, _f, _f, _p]
        L.oracle_core_fine_water_debug.argtypes = [_p, _p, _i, _i, _p, _p]
        L.oracle_core_inflow.argtypes = [_p, _i, _f, _f, _f]
        L.oracle_core_set_hydro_solids.argtypes = [_p, _p, _i]
        L.oracle_core_solid_mask.argtypes = [_p, _p]
        L.oracle_core_hydro_load.argtypes = [_p, _p]
        L.oracle_core_lay_slurry_on_water.argtypes = [_p, _f, _i]
        L.oracle_core_lay_slurry_on_water.restype = _f
    return L


def _ptr(a):
    return a.ctypes.data_as(_p) if a is not None else None


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Scratch:
    """Stands in for the reference's thread-local sheet scratch."""

    def __init__(self):
        self.h = lib().oracle_scratch_new()

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_scratch_free(self.h)
            self.h = None


def step_sheet(h, u, v, bed, nu, gate, res, cell, dt, vorticity, eps=1.0e-6, banks=False,
               sub_cap=8.0, pace=0, inner_par=True, scratch=None):
    """In-place `step_sheet_eps` (src/fluid_core.rs:856) on float32 arrays."""
    sc = scratch or Scratch()
    lib().oracle_step_sheet(_ptr(h), _ptr(u), _ptr(v), _ptr(bed), _ptr(nu), _ptr(gate), res, cell, dt,
                            vorticity, eps, int(banks), sub_cap, pace, int(inner_par), sc.h)


def transport_open(h, vel, gate, res, cell, dt, box, along_x, bed=None, frac_cap=0.45, serial=False):
    n = res * res
    removed = np.zeros(n, np.float32)
    added = np.zeros(n, np.float32)
    i0, i1, j0, j1 = box
    lib().oracle_transport_open(_ptr(h), _ptr(vel), _ptr(gate), res, cell, dt, i0, i1, j0, j1, int(along_x),
                                _ptr(bed), frac_cap, int(serial), _ptr(removed), _ptr(added))
    return removed, added


def sheet_work_boxes(h, res, eps, allow_split=True, flood=False):
    out = np.zeros(4 * 4096, np.int32)
    n = lib().oracle_sheet_work_boxes(_ptr(h), res, eps, int(allow_split), int(flood), _ptr(out), 4096)
    return [tuple(int(x) for x in out[4 * k:4 * k + 4]) for k in range(n)]


def awake_work_boxes(h, u, v, bed, res, cell, eps):
    out = np.zeros(4 * 4096, np.int32)
    n = lib().oracle_awake_work_boxes(_ptr(h), _ptr(u), _ptr(v), _ptr(bed), res, cell, eps, _ptr(out), 4096)
    return [tuple(int(x) for x in out[4 * k:4 * k + 4]) for k in range(n)]


def dynamic_viscosity(grain, moisture):
    return lib().oracle_dynamic_viscosity(grain, moisture)


def sheet_damp(nu):
    return lib().oracle_sheet_damp(nu)


def sheet_mobility_for(nu):
    return lib().oracle_sheet_mobility_for(nu)


def rut_heal(grain, moisture):
    out = np.zeros(4, np.float32)
    lib().oracle_rut_heal(grain, moisture, _ptr(out))
    return dict(level_s=float(out[0]), relief0=float(out[1]), relief_8s=float(out[2]),
                still_deep_at_8s=bool(out[3] > 0.5))


FIELDS = {"water": 0, "slurry": 1, "uw": 2, "vw": 3, "us": 4, "vs": 5, "bed": 6, "moisture": 7, "foam": 8,
          "turbid": 9, "susp": 10}
TRACER_BOOKS = ("suspended_m3", "settled_suspended_m3", "frozen_suspended_m3", "entrained_m3", "turbid_m3",
                "turbid_settled_m3", "stirred_m3", "frozen_turbid_m3")


class Core:
    """The reference `FluidCore` subset on the sheet path (window 200 at 0.2 m by default)."""

    _L = staticmethod(lib)
    _np = np.float32
    _Cfg, _Tire, _Spray = CoreCfg, Tire, Spray

    def _arr(self, a):
        return np.ascontiguousarray(a, dtype=self._np)

    def __init__(self, res=200, cell=0.2, fine_res=160, fine_cell=0.02, layout=0, tire_r=0.56,
                 soften=True, inner_par=False, center=(0.0, 0.0), threads=1):
        self.res = res
        self.fine_res = fine_res
        cfg = self._Cfg(res, cell, fine_res, fine_cell, layout, tire_r, int(soften), int(inner_par),
                      center[0], center[1], int(threads))
        self.h = self._L().oracle_core_new(ctypes.byref(cfg))

    def __del__(self):
        if getattr(self, "h", None):
            self._L().oracle_core_free(self.h)
            self.h = None

    def map_water_bed(self, bed, water):
        return self._L().oracle_core_map_water_bed(self.h, _ptr(self._arr(bed)), _ptr(self._arr(water)))

    def map_grain(self, grain):
        self._L().oracle_core_map_grain(self.h, _ptr(np.ascontiguousarray(grain, np.uint8)))

    def map_water_velocity(self, u, v):
        self._L().oracle_core_map_water_velocity(self.h, _ptr(self._arr(u)), _ptr(self._arr(v)))

    def pour_water(self, x0, x1, z0, z1, depth):
        return self._L().oracle_core_pour(self.h, x0, x1, z0, z1, depth, 1, 3, 1.0)

    def pour_slurry(self, x0, x1, z0, z1, depth, grain, moisture):
        return self._L().oracle_core_pour(self.h, x0, x1, z0, z1, depth, 0, grain, moisture)

    def lay_slurry_mask(self, depth, grain, moisture):
        return self._L().oracle_core_lay_slurry_mask(self.h, _ptr(self._arr(depth)), grain, moisture)

    def read_substrate(self, bed, moisture, grain):
        self._L().oracle_core_read_substrate(self.h, _ptr(self._arr(bed)), _ptr(self._arr(moisture)),
                                         _ptr(np.ascontiguousarray(grain, np.uint8)))

    def push_tire(self, **kw):
        t = self._Tire(kw["x"], kw["z"], kw.get("forward_x", 0.0), kw.get("forward_z", 1.0), kw["radius"],
                 kw["width"], kw["speed"], kw.get("slip", 0.0))
        self._L().oracle_core_push_tire(self.h, ctypes.byref(t))

    def step(self, dt):
        cap = 65536
        buf = (self._Spray * cap)()
        n = self._L().oracle_core_step(self.h, dt, buf, cap)
        return [(s.x, s.y, s.z, s.vx, s.vy, s.vz, s.volume, s.kind) for s in buf[:min(n, cap)]]

    def ledger(self):
        o = np.zeros(5, self._np)
        o64 = np.zeros(2, np.float64)
        self._L().oracle_core_ledger(self.h, _ptr(o), _ptr(o64))
        return dict(water_m3=float(o[0]), slurry_m3=float(o[1]), frozen_water_m3=float(o[2]),
                    frozen_slurry_m3=float(o[3]), spray_m3=float(o[4]), water64=float(o64[0]),
                    slurry64=float(o64[1]))

    def get(self, name):
        out = np.zeros(self.res * self.res, self._np)
        self._L().oracle_core_get(self.h, FIELDS[name], _ptr(out))
        return out

    def set(self, name, arr):
        self._L().oracle_core_set(self.h, FIELDS[name], _ptr(self._arr(arr)))

    def grain(self):
        out = np.zeros(self.res * self.res, np.uint8)
        self._L().oracle_core_get_grain(self.h, _ptr(out))
        return out

    def publish(self):
        film = np.zeros(2 * self.res * self.res, self._np)
        flow = np.zeros(4 * self.res * self.res, self._np)
        self._L().oracle_core_publish(self.h, _ptr(film), _ptr(flow))
        return film, flow

    def set_fine_pace(self, pace):
        self._L().oracle_core_set_fine_pace(self.h, pace)

    def set_turbidity_enabled(self, on):
        self._L().oracle_core_set_turbidity(self.h, int(on))

    def set_reach_turbidity(self, c):
        self._L().oracle_core_set_reach_turbidity(self.h, c)

    def tracer_books(self):
        """The tracer books: f32 as the reference keeps them, and '<name>64' in FP64."""
        o = np.zeros(8, self._np if self._np == np.float64 else np.float32)
        o64 = np.zeros(8, np.float64)
        self._L().oracle_core_tracer_books(self.h, _ptr(o), _ptr(o64))
        d = {k: float(v) for k, v in zip(TRACER_BOOKS, o)}
        d.update({k + "64": float(v) for k, v in zip(TRACER_BOOKS, o64)})
        return d

    def set_fine_sub_cap(self, cap):
        self._L().oracle_core_set_fine_sub_cap(self.h, cap)

    def set_near_field(self, on):
        self._L().oracle_core_set_near_field(self.h, int(on))

    def set_open_water(self, on, mobility=0.0, manning_n=0.0, eddy_m2_s=0.0):
        self._L().oracle_core_set_open_water(self.h, int(on), mobility, manning_n, eddy_m2_s)

    def set_surface_diffusion(self, m2_s):
        self._L().oracle_core_set_surface_diffusion(self.h, m2_s)

    def set_river_reach(self, reach):
        """reach: dict(along_z, positive, cross0, cross1, rows, inlet_eta, outlet_eta, inlet_speed_m_s[,
        inlet_turbidity]) or None."""
        r = reach or {}
        self._L().oracle_core_set_river_reach(self.h, int(reach is not None), int(r.get("along_z", False)),
                                          int(r.get("positive", True)), r.get("cross0", 0.0), r.get("cross1", 0.0),
                                          int(r.get("rows", 1)), r.get("inlet_eta", 0.0), r.get("outlet_eta", 0.0),
                                          r.get("inlet_speed_m_s", 0.0))
        self.set_reach_turbidity(r.get("inlet_turbidity", 0.0))

    def reach_bank_m3(self):
        return self._L().oracle_core_reach_bank(self.h)

    def set_wave_maker(self, wave):
        """wave: dict(x0, x1, z0, z1, dir_x, dir_z, amplitude_m_s, period_s, ramp_s) or None."""
        w = wave or {}
        self._L().oracle_core_set_wave_maker(self.h, int(wave is not None), w.get("x0", 0.0), w.get("x1", 0.0),
                                         w.get("z0", 0.0), w.get("z1", 0.0), w.get("dir_x", 0.0), w.get("dir_z", 0.0),
                                         w.get("amplitude_m_s", 0.0), w.get("period_s", 0.0), w.get("ramp_s", 0.0))

    def recenter(self, cx, cz):
        self._L().oracle_core_recenter(self.h, cx, cz)

    def origin(self):
        o = np.zeros(2, self._np)
        self._L().oracle_core_origin(self.h, _ptr(o))
        return float(o[0]), float(o[1])

    def parked_count(self):
        return self._L().oracle_core_parked_count(self.h)

    def near_tiles(self):
        return self._L().oracle_core_near_tiles(self.h)

    def spray_m3(self):
        return self._L().oracle_core_spray_m3(self.h)

    def non_finite_count(self):
        return self._L().oracle_core_non_finite(self.h)

    def sample(self, x, z):
        o = np.zeros(7, self._np)
        self._L().oracle_core_sample(self.h, x, z, _ptr(o))
        return dict(water_m=float(o[0]), slurry_m=float(o[1]), u=float(o[2]), v=float(o[3]),
                    moisture=float(o[5]), bed_m=float(o[6]))

    def fine_water_debug(self, tires, patch=0):
        arr = (self._Tire * len(tires))()
        for k, t in enumerate(tires):
            arr[k] = self._Tire(t["x"], t["z"], t.get("forward_x", 0.0), t.get("forward_z", 1.0), t["radius"],
                          t["width"], t["speed"], t.get("slip", 0.0))
        out = np.zeros(self.fine_res * self.fine_res, self._np)
        org = np.zeros(2, self._np)
        self._L().oracle_core_fine_water_debug(self.h, arr, len(tires), patch, _ptr(out), _ptr(org))
        return out, org

    SOLID_KEYS = ("x", "z", "yaw", "half_length", "half_width", "bottom_y", "top_y", "contact", "radius", "width")

    def set_hydro_solids(self, solids):
        """solids: dicts with the HydroSolid fields (src/fluid_core.rs:219-240)."""
        packed = np.array([[float(sd.get(k, 0.0)) for k in self.SOLID_KEYS] for sd in solids] or [[0.0] * 10],
                          self._np)
        self._L().oracle_core_set_hydro_solids(self.h, _ptr(packed), len(solids))

    LOAD_KEYS = ("force_x", "force_z", "buoyancy_n", "hull_buoyancy_n", "wheel_buoyancy_n", "displaced_m3",
                 "eroded_m3", "hole_m", "wheel_blocks", "belly_blocks")

    def lay_slurry_on_water(self, depth, grain):
        return self._L().oracle_core_lay_slurry_on_water(self.h, depth, grain)

    def hydro_load(self):
        o = np.zeros(10, self._np)
        self._L().oracle_core_hydro_load(self.h, _ptr(o))
        d = {k: float(v) for k, v in zip(self.LOAD_KEYS, o)}
        d["wheel_blocks"], d["belly_blocks"] = int(o[8]), int(o[9])
        return d

    def solid_mask(self):
        out = np.zeros(self.res * self.res, np.uint8)
        self._L().oracle_core_solid_mask(self.h, _ptr(out))
        return out

    def set_inflow(self, j, x0, x1, rate_m3_s):
        self._L().oracle_core_inflow(self.h, j, x0, x1, rate_m3_s)


class CoreRN(Core):
    """The same step with e^x, x^y and hypot as the double result rounded
    once to float, the device's forms (liboracle_silt_rn). The C library's
    expf differs from that on ~1e-4 of inputs; where such a 1-ulp factor is
    absorbed by the f32 update the planes stay equal but an FP64 book moves,
    and this build shows which."""

    _L = staticmethod(lib_rn)


class Core64(Core):
    """The same FluidCore subset computed in FP64 throughout (liboracle_silt_f64):
    the nested-sheet oracle that the learned closure's flux and depth errors
    are stated against. Fields come back as float64."""

    _L = staticmethod(lib64)
    _np = np.float64
    _Cfg, _Tire, _Spray = CoreCfg64, Tire64, Spray64
