"""Python binding of libsilt_b200.so, the B200 sheet step behind its C ABI
(include/silt_sheet.h).

`Sheet` mirrors the reference's `FluidCore` surface on the sheet path
(x3-team/Dirty-gen src/fluid_core.rs): seeding, push_tire, step, ledger,
coarse_cell, export_maps and the render-contract film/flow publish. There is
no CPU fallback: loading fails loudly when the CUDA library is missing.
"""
import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsilt_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "silt_sheet.h")

SILT_OK, SILT_OK_NOOP, SILT_EINVAL, SILT_ECUDA, SILT_ETIMEOUT, SILT_ENOMEM, SILT_EBOUND = 0, 1, -1, -2, -3, -4, -5
CLAY, SILT, SAND, WATER, OTHER = 0, 1, 2, 3, 4
FINE_MEAN_PATCH, FINE_PER_TIRE = 0, 1
ENGINE_AUTO, ENGINE_WINDOW, ENGINE_GRID = 0, 1, 2
CONFINE_SWEEP, CONFINE_SNAPSHOT = 0, 1

_f = ctypes.c_float
_i = ctypes.c_int32
_p = ctypes.c_void_p


class Cfg(ctypes.Structure):
    _fields_ = [("res", _i), ("cell", _f), ("fine_res", _i), ("fine_cell", _f), ("fine_layout", _i),
                ("tire_r", _f), ("soften_border", _i), ("center_x", _f), ("center_z", _f), ("device", _i),
                ("stream", _p), ("engine", _i)]


class TirePush(ctypes.Structure):
    _fields_ = [(k, _f) for k in ("x", "z", "forward_x", "forward_z", "radius", "width", "speed", "slip")]


class SprayEvent(ctypes.Structure):
    _fields_ = [(k, _f) for k in ("x", "y", "z", "vx", "vy", "vz", "volume")] + [("kind", _i)]


class Ledger(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("water_m3", "slurry_m3", "frozen_water_m3", "frozen_slurry_m3",
                                               "spray_m3", "opened_m3", "total_m3", "cut_m3", "reach_m3",
                                               "round_m3", "suspended_m3", "settled_suspended_m3",
                                               "frozen_suspended_m3", "entrained_m3", "turbid_m3",
                                               "turbid_settled_m3", "frozen_turbid_m3", "stirred_m3")]


class RiverReach(ctypes.Structure):
    _fields_ = [("along_z", _i), ("positive", _i), ("cross0", _f), ("cross1", _f), ("rows", _i),
                ("inlet_eta", _f), ("outlet_eta", _f), ("inlet_speed_m_s", _f), ("inlet_turbidity", _f)]


class WaveMaker(ctypes.Structure):
    _fields_ = [(k, _f) for k in ("x0", "x1", "z0", "z1", "dir_x", "dir_z", "amplitude_m_s", "period_s", "ramp_s")]


class HydroSolid(ctypes.Structure):
    _fields_ = [(k, _f) for k in ("x", "z", "yaw", "half_length", "half_width", "bottom_y", "top_y")] + \
               [("contact", _i), ("radius", _f), ("width", _f)]


class HydroLoad(ctypes.Structure):
    _fields_ = [(k, _f) for k in ("force_x", "force_z", "buoyancy_n", "hull_buoyancy_n", "wheel_buoyancy_n",
                                  "displaced_m3", "eroded_m3", "hole_m")] + \
               [("wheel_blocks", ctypes.c_uint32), ("belly_blocks", ctypes.c_uint32)]


class GroundSample(ctypes.Structure):
    _fields_ = [(k, _f) for k in ("water_m", "slurry_m", "u", "v", "settled_dust_m", "moisture", "bed_m")]


class CoarseCell(ctypes.Structure):
    _fields_ = [(k, _f) for k in ("x", "z", "bed_m", "water_m", "slurry_m", "moisture", "u", "v", "turbidity")]


class StepParts(ctypes.Structure):
    _fields_ = [("force_ms", ctypes.c_double), ("transport_ms", ctypes.c_double), ("fine_ms", ctypes.c_double),
                ("steps", ctypes.c_int64), ("launches", ctypes.c_int64), ("force_launches", ctypes.c_int64),
                ("force_cells", ctypes.c_int64), ("force_cells_water", ctypes.c_int64),
                ("device_counts", ctypes.c_int64), ("host_step_ms", ctypes.c_double),
                ("host_fine_ms", ctypes.c_double), ("sweep_launches", ctypes.c_int64),
                ("sweep_passes_max", ctypes.c_int64), ("sweep_fallbacks", ctypes.c_int64),
                ("sweep_solves", ctypes.c_int64), ("sweep_local_passes", ctypes.c_int64),
                ("host_phase_ms", ctypes.c_double * 8)]


class BatchTune(ctypes.Structure):
    _fields_ = [("sweep_ctas_per_sm", _i), ("transport_blocks", _i), ("tracer_blocks", _i), ("tuned", _i),
                ("trials", _i), ("trial_ms", ctypes.c_float * 16)]


def parts_dict(sp):
    """A StepParts as a dict (arrays as lists)."""
    out = {}
    for k, _ in StepParts._fields_:
        v = getattr(sp, k)
        out[k] = list(v) if isinstance(v, ctypes.Array) else v
    return out


class KernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 96), ("launches", ctypes.c_int64), ("ms", ctypes.c_double)]


class SiltError(RuntimeError):
    pass


_lib = None


def header_functions():
    """Names of every function include/silt_sheet.h declares."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|size_t|const char\*)\s+(silt_\w+)\s*\(", text, re.M)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SiltError(f"{LIB_PATH} is missing: build it with `make -C dirty-gen_b200` (no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.silt_last_error.restype = ctypes.c_char_p
        L.silt_cfg_default.argtypes = [ctypes.POINTER(Cfg)]
        L.silt_cfg_default.restype = None
        L.silt_sheet_create.argtypes = [ctypes.POINTER(Cfg), ctypes.POINTER(_p)]
        for name, args in {
            "silt_sheet_destroy": [_p], "silt_sheet_sync": [_p],
            "silt_map_water_bed": [_p, _p, _p, _p], "silt_map_grain": [_p, _p],
            "silt_map_water_velocity": [_p, _p, _p],
            "silt_pour_water": [_p, _f, _f, _f, _f, _f, _p],
            "silt_pour_slurry": [_p, _f, _f, _f, _f, _f, _i, _f, _p],
            "silt_lay_slurry_mask": [_p, _p, _i, _f, _p],
            "silt_read_substrate_grid": [_p, _p, _p, _p],
            "silt_set_inflow": [_p, _i, _f, _f, _f],
            "silt_push_tire": [_p, ctypes.POINTER(TirePush)],
            "silt_step": [_p, _f, _p, _i, ctypes.POINTER(_i)],
            "silt_get_ledger": [_p, ctypes.POINTER(Ledger)],
            "silt_get_coarse_cell": [_p, _i, _i, ctypes.POINTER(CoarseCell)],
            "silt_export_maps": [_p, _p, _p, _p, _p],
            "silt_publish_film_flow": [_p, _p, _p],
            "silt_publish_film_flow_device": [_p, _p, _p],
            "silt_non_finite_count": [_p, ctypes.POINTER(ctypes.c_uint32)],
            "silt_spray_m3": [_p, ctypes.POINTER(ctypes.c_double)],
            "silt_window_bounds": [_p, _p, _p, _p],
            "silt_read_plane": [_p, _i, _p], "silt_write_plane": [_p, _i, _p],
            "silt_fine_water_debug": [_p, _p, _i, _i, _p, _p],
            "silt_near_tiles": [_p, ctypes.POINTER(_i)],
            "silt_set_fine_sub_cap": [_p, _f], "silt_set_fine_pace": [_p, _i], "silt_set_near_field": [_p, _i],
            "silt_set_confinement": [_p, _i],
            "silt_step_sheet": [_p, _p, _p, _p, _p, _p, _i, _f, _f, _f, _p, _p],
            "silt_set_step_timing": [_p, _i], "silt_get_step_parts": [_p, ctypes.POINTER(StepParts)],
            "silt_step_sheet_noalloc": [_p, _p, _p, _p, _p, _p, _i, _f, _f, _f, _p],
            "silt_batch_create": [ctypes.POINTER(_p), _i, ctypes.POINTER(_p)],
            "silt_batch_destroy": [_p], "silt_batch_step": [_p, _f],
            "silt_batch_get_ledgers": [_p, ctypes.POINTER(Ledger)],
            "silt_batch_push_tires": [_p, _p, ctypes.POINTER(TirePush), _i],
            "silt_batch_set_timing": [_p, _i], "silt_batch_get_parts": [_p, ctypes.POINTER(StepParts)],
            "silt_batch_autotune": [_p, _i], "silt_batch_get_tune": [_p, ctypes.POINTER(BatchTune)],
            "silt_batch_set_tune": [_p, ctypes.POINTER(BatchTune)],
            "silt_plane_device": [_p, _i, ctypes.POINTER(_p)], "silt_sheet_copy_state": [_p, _p],
            "silt_set_open_water": [_p, _i, _f, _f, _f], "silt_set_surface_diffusion": [_p, _f],
            "silt_set_turbidity_enabled": [_p, _i], "silt_sample": [_p, _f, _f, ctypes.POINTER(GroundSample)],
            "silt_recenter": [_p, _f, _f], "silt_set_center": [_p, _f, _f],
            "silt_set_river_reach": [_p, ctypes.POINTER(RiverReach)],
            "silt_set_wave_maker": [_p, ctypes.POINTER(WaveMaker)],
            "silt_check_fixed_division": [_f, ctypes.POINTER(ctypes.c_ulonglong), _p],
            "silt_known_exact_divisors": [_p, _i],
            "silt_set_kernel_timing": [_i], "silt_get_kernel_times": [_p, _i, ctypes.POINTER(_i)],
            "silt_set_hydro_solids": [_p, ctypes.POINTER(HydroSolid), _i],
            "silt_get_hydro_load": [_p, ctypes.POINTER(HydroLoad)],
            "silt_lay_slurry_on_water": [_p, _f, _i, _p], "silt_window_origin": [_f, _f, _i, _f, _p],
        }.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.silt_step_sheet_scratch_bytes.argtypes = [_i]
        L.silt_step_sheet_scratch_bytes.restype = ctypes.c_size_t
        _lib = L
    return _lib


def check(rc, what=""):
    if rc < 0:
        raise SiltError(f"{what}: rc={rc} {lib().silt_last_error().decode()}")
    return rc


def _ptr(a):
    return a.ctypes.data_as(_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


PLANES = {"water": 0, "slurry": 1, "uw": 2, "vw": 3, "us": 4, "vs": 5, "bed": 6, "moisture": 7, "foam": 8,
          "turbid": 9, "susp": 10}


# A tire push as a numpy record (the layout of silt_tire_push).
TIRE_DTYPE = np.dtype([("x", np.float32), ("z", np.float32), ("forward_x", np.float32), ("forward_z", np.float32),
                       ("radius", np.float32), ("width", np.float32), ("speed", np.float32), ("slip", np.float32)])


def make_push(t):
    return TirePush(t["x"], t["z"], t.get("forward_x", 0.0), t.get("forward_z", 1.0), t["radius"], t["width"],
                    t["speed"], t.get("slip", 0.0))


class _DeviceArray:
    """A device FP32 array exposed through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class Sheet:
    """A window of the two-layer sheet on the GPU (FluidCore, src/fluid_core.rs:4808)."""

    def __init__(self, res=200, cell=0.2, fine_res=160, fine_cell=0.02, layout=FINE_MEAN_PATCH, tire_r=0.56,
                 soften=True, center=(0.0, 0.0), device=0, stream=None, engine=ENGINE_AUTO):
        L = lib()
        cfg = Cfg()
        L.silt_cfg_default(ctypes.byref(cfg))
        cfg.res, cfg.cell, cfg.fine_res, cfg.fine_cell = res, cell, fine_res, fine_cell
        cfg.fine_layout, cfg.tire_r, cfg.soften_border = layout, tire_r, int(soften)
        cfg.center_x, cfg.center_z, cfg.device = center[0], center[1], device
        cfg.stream = stream
        cfg.engine = engine
        h = _p()
        check(L.silt_sheet_create(ctypes.byref(cfg), ctypes.byref(h)), "silt_sheet_create")
        self.h = h
        self._destroy = L.silt_sheet_destroy  # kept: at interpreter exit the module's globals may be gone
        self.res = res
        self.fine_res = fine_res
        self.device = device

    def close(self):
        h = getattr(self, "h", None)
        if h:
            self.h = None
            self._destroy(h)

    __del__ = close

    def sync(self):
        check(lib().silt_sheet_sync(self.h), "sync")

    def map_water_bed(self, bed, water):
        vol = _f(0)
        check(lib().silt_map_water_bed(self.h, _ptr(_f32(bed)), _ptr(_f32(water)), ctypes.byref(vol)), "map_water_bed")
        return vol.value

    def map_grain(self, grain):
        check(lib().silt_map_grain(self.h, _ptr(np.ascontiguousarray(grain, np.uint8))), "map_grain")

    def map_water_velocity(self, u, v):
        check(lib().silt_map_water_velocity(self.h, _ptr(_f32(u)), _ptr(_f32(v))), "map_water_velocity")

    def pour_water(self, x0, x1, z0, z1, depth):
        vol = _f(0)
        check(lib().silt_pour_water(self.h, x0, x1, z0, z1, depth, ctypes.byref(vol)), "pour_water")
        return vol.value

    def pour_slurry(self, x0, x1, z0, z1, depth, grain, moisture):
        vol = _f(0)
        check(lib().silt_pour_slurry(self.h, x0, x1, z0, z1, depth, grain, moisture, ctypes.byref(vol)), "pour_slurry")
        return vol.value

    def lay_slurry_mask(self, depth, grain, moisture):
        vol = _f(0)
        check(lib().silt_lay_slurry_mask(self.h, _ptr(_f32(depth)), grain, moisture, ctypes.byref(vol)), "lay_slurry")
        return vol.value

    def read_substrate(self, bed, moisture, grain):
        check(lib().silt_read_substrate_grid(self.h, _ptr(_f32(bed)), _ptr(_f32(moisture)),
                                             _ptr(np.ascontiguousarray(grain, np.uint8))), "read_substrate_grid")

    def set_inflow(self, j, x0, x1, rate_m3_s):
        check(lib().silt_set_inflow(self.h, j, x0, x1, rate_m3_s), "set_inflow")

    def push_tire(self, **t):
        p = make_push(t)
        check(lib().silt_push_tire(self.h, ctypes.byref(p)), "push_tire")

    def step(self, dt, want_spray=True, cap=8192):
        if not want_spray:
            check(lib().silt_step(self.h, dt, None, 0, None), "step")
            return None
        if getattr(self, "_spray_buf", None) is None or len(self._spray_buf) < cap:
            self._spray_buf = (SprayEvent * cap)()
        n = _i(0)
        buf = self._spray_buf
        check(lib().silt_step(self.h, dt, buf, cap, ctypes.byref(n)), "step")
        return [(e.x, e.y, e.z, e.vx, e.vy, e.vz, e.volume, e.kind) for e in buf[:min(n.value, cap)]]

    def ledger(self):
        led = Ledger()
        check(lib().silt_get_ledger(self.h, ctypes.byref(led)), "ledger")
        return {k: getattr(led, k) for k, _ in Ledger._fields_}

    def coarse_cell(self, i, j):
        c = CoarseCell()
        rc = check(lib().silt_get_coarse_cell(self.h, i, j, ctypes.byref(c)), "coarse_cell")
        return None if rc == SILT_OK_NOOP else {k: getattr(c, k) for k, _ in CoarseCell._fields_}

    def get(self, name):
        out = np.zeros(self.res * self.res, np.float32)
        check(lib().silt_read_plane(self.h, PLANES[name], _ptr(out)), "read_plane")
        return out

    def set(self, name, arr):
        check(lib().silt_write_plane(self.h, PLANES[name], _ptr(_f32(arr))), "write_plane")

    def plane_device(self, name):
        """The plane's device memory as a torch tensor view (res x res FP32),
        valid until the next step or write; read it on the sheet's stream."""
        import torch

        ptr = ctypes.c_void_p()
        check(lib().silt_plane_device(self.h, PLANES[name], ctypes.byref(ptr)), "plane_device")
        view = _DeviceArray(ptr.value, (self.res, self.res))
        return torch.as_tensor(view, device=f"cuda:{self.device}")

    def copy_state_from(self, other):
        check(lib().silt_sheet_copy_state(self.h, other.h), "copy_state")

    def set_open_water(self, on, mobility=0.0, manning_n=0.0, eddy_m2_s=0.0):
        """FluidCore::set_open_water (on=False is None)."""
        check(lib().silt_set_open_water(self.h, int(on), mobility, manning_n, eddy_m2_s), "set_open_water")

    def set_surface_diffusion(self, m2_s):
        check(lib().silt_set_surface_diffusion(self.h, m2_s), "set_surface_diffusion")

    def recenter(self, cx, cz):
        """FluidCore::recenter: move the window; cells that leave are parked, cells that enter restored."""
        check(lib().silt_recenter(self.h, cx, cz), "recenter")

    def set_center(self, cx, cz):
        check(lib().silt_set_center(self.h, cx, cz), "set_center")

    def origin(self):
        return self.window_bounds()[:2]

    def window_bounds(self):
        """FluidCore::window_bounds: origin x, origin z, extent (m)."""
        ox, oz, ext = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        check(lib().silt_window_bounds(self.h, ctypes.byref(ox), ctypes.byref(oz), ctypes.byref(ext)), "window_bounds")
        return ox.value, oz.value, ext.value

    def set_river_reach(self, reach):
        """FluidCore::set_river_reach: dict of RiverReach fields, or None."""
        if reach is None:
            check(lib().silt_set_river_reach(self.h, None), "set_river_reach")
            return
        r = RiverReach(int(reach.get("along_z", False)), int(reach.get("positive", True)), reach.get("cross0", 0.0),
                       reach.get("cross1", 0.0), int(reach.get("rows", 1)), reach.get("inlet_eta", 0.0),
                       reach.get("outlet_eta", 0.0), reach.get("inlet_speed_m_s", 0.0),
                       reach.get("inlet_turbidity", 0.0))
        check(lib().silt_set_river_reach(self.h, ctypes.byref(r)), "set_river_reach")

    def set_hydro_solids(self, solids):
        """FluidCore::set_hydro_solids: dicts with the HydroSolid fields (x, z,
        yaw, half_length, half_width, bottom_y, top_y, contact, radius, width);
        an empty list removes the walls."""
        arr = (HydroSolid * max(len(solids), 1))()
        for k, sd in enumerate(solids):
            arr[k] = HydroSolid(*[float(sd.get(n, 0.0)) for n in ("x", "z", "yaw", "half_length", "half_width",
                                                                   "bottom_y", "top_y")],
                                int(bool(sd.get("contact", False))), float(sd.get("radius", 0.0)),
                                float(sd.get("width", 0.0)))
        check(lib().silt_set_hydro_solids(self.h, arr, len(solids)), "set_hydro_solids")

    def lay_slurry_on_water(self, depth, grain):
        """FluidCore::lay_slurry_on_water: returns the laid volume (f32)."""
        vol = ctypes.c_float(0.0)
        check(lib().silt_lay_slurry_on_water(self.h, float(depth), int(grain), ctypes.byref(vol)),
              "lay_slurry_on_water")
        return vol.value

    def hydro_load(self):
        """FluidCore::hydro_load: forces, buoyancy and scour as a dict."""
        o = HydroLoad()
        check(lib().silt_get_hydro_load(self.h, ctypes.byref(o)), "hydro_load")
        return {k: getattr(o, k) for k, _ in HydroLoad._fields_}

    def set_wave_maker(self, wave):
        """FluidCore::set_wave_maker: dict of WaveMaker fields, or None."""
        if wave is None:
            check(lib().silt_set_wave_maker(self.h, None), "set_wave_maker")
            return
        w = WaveMaker(*[wave.get(k, 0.0) for k, _ in WaveMaker._fields_])
        check(lib().silt_set_wave_maker(self.h, ctypes.byref(w)), "set_wave_maker")

    def set_turbidity_enabled(self, on):
        check(lib().silt_set_turbidity_enabled(self.h, int(on)), "set_turbidity_enabled")

    def sample(self, x, z):
        """FluidCore::sample between steps: the coarse cell under (x, z), None outside."""
        g = GroundSample()
        rc = check(lib().silt_sample(self.h, x, z, ctypes.byref(g)), "sample")
        return None if rc == SILT_OK_NOOP else {k: getattr(g, k) for k, _ in GroundSample._fields_}

    def export_maps(self):
        n = self.res * self.res
        out = [np.zeros(n, np.float32) for _ in range(4)]
        check(lib().silt_export_maps(self.h, *[_ptr(o) for o in out]), "export_maps")
        return dict(zip(("height", "vel_u", "vel_v", "moisture"), out))

    def publish(self):
        film = np.zeros(2 * self.res * self.res, np.float32)
        flow = np.zeros(4 * self.res * self.res, np.float32)
        check(lib().silt_publish_film_flow(self.h, _ptr(film), _ptr(flow)), "publish")
        return film, flow

    def non_finite_count(self):
        c = ctypes.c_uint32(0)
        check(lib().silt_non_finite_count(self.h, ctypes.byref(c)), "non_finite_count")
        return c.value

    def spray_m3(self):
        d = ctypes.c_double(0)
        check(lib().silt_spray_m3(self.h, ctypes.byref(d)), "spray_m3")
        return d.value

    def set_fine_pace(self, pace):
        check(lib().silt_set_fine_pace(self.h, pace), "set_fine_pace")

    def set_fine_sub_cap(self, cap):
        check(lib().silt_set_fine_sub_cap(self.h, cap), "set_fine_sub_cap")

    def set_near_field(self, on):
        check(lib().silt_set_near_field(self.h, int(on)), "set_near_field")

    def set_confinement(self, form):
        """CONFINE_SWEEP (the reference step pair's Gauss-Seidel sweep, the
        default) or CONFINE_SNAPSHOT (the Jacobi form) on the grid engine."""
        check(lib().silt_set_confinement(self.h, int(form)), "set_confinement")

    def near_tiles(self):
        c = _i(0)
        check(lib().silt_near_tiles(self.h, ctypes.byref(c)), "near_tiles")
        return c.value

    def set_step_timing(self, on):
        check(lib().silt_set_step_timing(self.h, int(on)), "set_step_timing")

    def step_parts(self):
        sp = StepParts()
        check(lib().silt_get_step_parts(self.h, ctypes.byref(sp)), "step_parts")
        return parts_dict(sp)

    def fine_water_debug(self, tires, patch=0):
        arr = (TirePush * max(len(tires), 1))()
        for k, t in enumerate(tires):
            arr[k] = make_push(t)
        out = np.zeros(self.fine_res * self.fine_res, np.float32)
        org = np.zeros(2, np.float32)
        check(lib().silt_fine_water_debug(self.h, arr, len(tires), patch, _ptr(out), _ptr(org)), "fine_water_debug")
        return out, org


def step_sheet_device(h, u, v, bed, nu, gate, res, cell, dt, vorticity, scratch, stream=None):
    """The free one-sheet operator on device pointers (ints)."""
    return check(lib().silt_step_sheet(h, u, v, bed, nu, gate, res, cell, dt, vorticity, scratch, stream),
                 "step_sheet")


def window_origin(center, res=200, cell=0.2):
    """FluidCore::window_origin: the snapped minimum corner of a window."""
    o = (ctypes.c_float * 2)()
    check(lib().silt_window_origin(float(center[0]), float(center[1]), int(res), float(cell), o), "window_origin")
    return float(o[0]), float(o[1])


def set_kernel_timing(on):
    """Per-launch device timing of every library kernel (process-wide)."""
    check(lib().silt_set_kernel_timing(int(on)), "set_kernel_timing")


def kernel_times():
    """Totals by kernel since timing was switched on: [{name, launches, ms}],
    largest total first. Waits for the device."""
    n = _i(0)
    check(lib().silt_get_kernel_times(None, 0, ctypes.byref(n)), "kernel_times")
    rows = (KernelTime * max(n.value, 1))()
    check(lib().silt_get_kernel_times(ctypes.cast(rows, _p), n.value, ctypes.byref(n)), "kernel_times")
    return [dict(name=r.name.decode(), launches=int(r.launches), ms=float(r.ms)) for r in rows[:n.value]]


def known_exact_divisors():
    """The divisors the library takes as checked without running the check."""
    n = lib().silt_known_exact_divisors(None, 0)
    out = np.zeros(max(n, 1), np.float32)
    check(lib().silt_known_exact_divisors(_ptr(out), n), "known_exact_divisors")
    return [float(x) for x in out[:n]]


def check_fixed_division(d, stream=None):
    """Mismatch counts of the grid engine's fixed-divisor division by d against
    IEEE division over every float x: (all, x zero, x subnormal, x inf/NaN,
    subnormal or zero quotient, rest)."""
    counts = (ctypes.c_ulonglong * 6)()
    check(lib().silt_check_fixed_division(float(d), counts, stream), "check_fixed_division")
    return tuple(int(c) for c in counts)


class Batch:
    """Many windows stepped together: each Sheet (grid engine, one stream) keeps
    its own state; step() advances them all, the coarse pairs through shared
    launches (silt_batch_step)."""

    def __init__(self, sheets):
        self.sheets = list(sheets)
        arr = (_p * len(self.sheets))(*[sh.h for sh in self.sheets])
        h = _p()
        check(lib().silt_batch_create(arr, len(self.sheets), ctypes.byref(h)), "batch_create")
        self.h = h
        self._destroy = lib().silt_batch_destroy

    def autotune(self, on=True):
        """Times the next steps under each candidate launch setting and keeps
        the fastest (silt_batch_autotune); every setting gives the same bits."""
        check(lib().silt_batch_autotune(self.h, int(on)), "batch_autotune")

    def tune(self):
        t = BatchTune()
        check(lib().silt_batch_get_tune(self.h, ctypes.byref(t)), "batch_get_tune")
        return {"sweep_ctas_per_sm": t.sweep_ctas_per_sm, "transport_blocks": t.transport_blocks,
                "tracer_blocks": t.tracer_blocks, "tuned": bool(t.tuned), "trials": t.trials,
                "trial_ms": [round(float(x), 4) for x in t.trial_ms[:min(t.trials, 16)]]}

    def set_tune(self, sweep_ctas_per_sm=0, transport_blocks=0, tracer_blocks=0):
        t = BatchTune(sweep_ctas_per_sm, transport_blocks, tracer_blocks, 0, 0)
        check(lib().silt_batch_set_tune(self.h, ctypes.byref(t)), "batch_set_tune")

    def close(self):
        h = getattr(self, "h", None)
        if h:
            self.h = None
            self._destroy(h)

    __del__ = close

    def step(self, dt):
        return check(lib().silt_batch_step(self.h, dt), "batch_step")

    def push_tires(self, windows, tires):
        """Tire pushes for many windows: tires[k] goes to window windows[k]. `tires` is a
        list of dicts as for Sheet.push_tire, or a numpy array of dtype TIRE_DTYPE."""
        n = len(tires)
        if n == 0:
            return
        idx = np.ascontiguousarray(windows, dtype=np.int32)
        if isinstance(tires, np.ndarray):
            rec = np.ascontiguousarray(tires, dtype=TIRE_DTYPE)
            arr = rec.ctypes.data_as(ctypes.POINTER(TirePush))
        else:
            arr = (TirePush * n)(*[make_push(t) for t in tires])
        check(lib().silt_batch_push_tires(self.h, _ptr(idx), arr, n), "batch_push_tires")

    def ledgers(self):
        arr = (Ledger * len(self.sheets))()
        check(lib().silt_batch_get_ledgers(self.h, arr), "batch_ledgers")
        return [{k: getattr(x, k) for k, _ in Ledger._fields_} for x in arr]

    def ledger_rows(self):
        """Every window's ledger as one FP64 array (a row per window), columns
        in the silt_ledger field order."""
        arr = (Ledger * len(self.sheets))()
        check(lib().silt_batch_get_ledgers(self.h, arr), "batch_ledgers")
        return np.frombuffer(arr, dtype=np.float64).reshape(len(self.sheets), len(Ledger._fields_)).copy()

    def set_timing(self, on):
        check(lib().silt_batch_set_timing(self.h, int(on)), "batch_set_timing")

    def parts(self):
        sp = StepParts()
        check(lib().silt_batch_get_parts(self.h, ctypes.byref(sp)), "batch_parts")
        return parts_dict(sp)
