"""Building crp_plan_desc structures (include/crp_gpu.h) from Python values.

A `ChainSpec` holds the field components and the module chain in ModuleList
order; `desc()` returns the ctypes PlanDesc view and keeps every array it
points into alive for as long as the spec lives.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _abi


def _v3(v) -> tuple:
    v = tuple(float(x) for x in (v if hasattr(v, "__len__") else (v, v, v)))
    if len(v) != 3:
        raise ValueError("expected a 3-vector")
    return v


@dataclass
class GridField:
    """MagneticFieldGrid over a Grid3f (MagneticFieldGrid.cpp:17)."""
    values: np.ndarray            # (nx, ny, nz, 3) float32, z fastest (Grid.h:338)
    origin: Sequence[float] = (0.0, 0.0, 0.0)
    spacing: Sequence[float] = (1.0, 1.0, 1.0)
    reflective: bool = False
    clip_volume: bool = False
    periodic: Optional[tuple] = None  # (origin, extends, reflective) PeriodicMagneticField
    interpolation: int = _abi.INTERPOLATION_TRILINEAR  # Grid::setInterpolationType (Grid.h:255)


@dataclass
class ScalarGrid:
    """A Grid1f (Grid.h:587): values (nx, ny, nz) float32, z fastest."""
    values: np.ndarray
    origin: Sequence[float] = (0.0, 0.0, 0.0)
    spacing: Sequence[float] = (1.0, 1.0, 1.0)
    reflective: bool = True  # what ModulatedMagneticFieldGrid's constructor sets (MagneticFieldGrid.cpp:23)
    clip_volume: bool = False
    interpolation: int = _abi.INTERPOLATION_TRILINEAR


@dataclass
class ModulatedGridField:
    """ModulatedMagneticFieldGrid (MagneticFieldGrid.cpp:51): the Grid3f field
    times the interpolated Grid1f modulation.  The constructor makes the
    Grid3f periodic and the modulation reflective (MagneticFieldGrid.cpp:22-23);
    setReflective(grid, modulation) is the two grids' own flags here."""
    grid: GridField
    modulation: ScalarGrid
    periodic: Optional[tuple] = None


@dataclass
class JF12Field:
    """JF12Field (variant JF12_VARIANT_JF12, JF12Field.cpp:8),
    PlanckJF12bField (JF12_VARIANT_PLANCK, :352) or JF12FieldSolenoidal
    (JF12_VARIANT_SOLENOIDAL, JF12FieldSolenoidal.cpp:8): the regular disk,
    toroidal halo and X fields, optionally striated (a Grid1f read by nearest
    value, setStriatedGrid, :113) and turbulent (a Grid3f scaled by the
    modelled strength, setTurbulentGrid, :118).  Giving a grid switches its
    part on, as the setters do; use_striated / use_turbulent override that.
    For JF12FieldSolenoidal, delta and zs are the constructor's arguments
    (the disk's transition width and the X field's scale height, metres;
    None: 3 kpc and 0.5 kpc) and outer_transition=False stands for
    deactivateOuterTransition()."""
    variant: int = _abi.JF12_VARIANT_JF12
    use_regular: bool = True
    use_disk: bool = True
    use_toroidal_halo: bool = True
    use_x: bool = True
    striated: Optional[ScalarGrid] = None
    turbulent: Optional[GridField] = None
    use_striated: Optional[bool] = None
    use_turbulent: Optional[bool] = None
    periodic: Optional[tuple] = None
    delta: Optional[float] = None
    zs: Optional[float] = None
    outer_transition: bool = True

    @staticmethod
    def defaults(variant=_abi.JF12_VARIANT_JF12) -> "_abi.JF12Desc":
        """The constructor's parameters (crp_jf12_defaults)."""
        d = _abi.JF12Desc()
        _abi.check(_abi.load().crp_jf12_defaults(int(variant), C.byref(d)))
        return d

    def parameters(self) -> "_abi.JF12Desc":
        """The constructor's parameters with this object's solenoidal
        arguments and setters applied (crp_jf12_solenoidal)."""
        d = self.defaults(self.variant)
        if self.variant == _abi.JF12_VARIANT_SOLENOIDAL:
            if self.delta is not None or self.zs is not None:
                delta = 3 * d.kpc if self.delta is None else float(self.delta)
                zs = 0.5 * d.kpc if self.zs is None else float(self.zs)
                _abi.check(_abi.load().crp_jf12_solenoidal(delta, zs, C.byref(d)))
            if not self.outer_transition:
                d.r2s = d.r2  # JF12FieldSolenoidal::deactivateOuterTransition (JF12FieldSolenoidal.cpp:89)
        elif self.delta is not None or self.zs is not None or not self.outer_transition:
            raise ValueError("JF12Field: delta, zs and outer_transition belong to JF12FieldSolenoidal")
        return d


@dataclass
class UF23Field:
    """UF23Field(model) (UF23Field.cpp:59): one of the eight coherent field
    models of Unger & Farrar 2023 (model: UF23_BASE ... UF23_NEBCOR, the
    order of UF23Field::ModelType)."""
    model: int = _abi.UF23_BASE
    periodic: Optional[tuple] = None

    @staticmethod
    def defaults(model=_abi.UF23_BASE) -> "_abi.UF23Desc":
        """The constructor's parameters (crp_uf23_defaults)."""
        d = _abi.UF23Desc()
        _abi.check(_abi.load().crp_uf23_defaults(int(model), C.byref(d)))
        return d


@dataclass
class PT11Field:
    """PT11Field() (PT11Field.cpp:8), the field of Pshirkov et al. 2011, with
    its switches: the ASS disk (the default) or the BSS disk, and the halo.
    As in the reference, switching one disk on switches the other off and
    sets its pitch and southern halo strength (setUseASS / setUseBSS,
    PT11Field.cpp:35-64); both on is an error."""
    use_ass: bool = True
    use_bss: bool = False
    use_halo: bool = True
    periodic: Optional[tuple] = None

    def desc(self) -> "_abi.PT11Desc":
        """The reference's state after PT11Field() and the setters that give
        these switches (crp_pt11_defaults, crp_pt11_use)."""
        if self.use_ass and self.use_bss:
            raise ValueError("PT11Field: the ASS and BSS disks exclude each other")
        lib, d = _abi.load(), _abi.PT11Desc()
        _abi.check(lib.crp_pt11_defaults(C.byref(d)))
        if self.use_bss:
            _abi.check(lib.crp_pt11_use(C.byref(d), _abi.PT11_BSS, 1))
        elif not self.use_ass:
            _abi.check(lib.crp_pt11_use(C.byref(d), _abi.PT11_ASS, 0))
        if not self.use_halo:
            _abi.check(lib.crp_pt11_use(C.byref(d), _abi.PT11_HALO, 0))
        return d


@dataclass
class TF17Field:
    """TF17Field(disk, halo) (TF17Field.cpp:10), the field of Terral &
    Ferriere 2017: disk model Ad1 (the default), Bd1 or Dd1 and halo model C0
    or C1 (the default), with setUseDiskField / setUseHaloField."""
    disk: int = _abi.TF17_AD1
    halo: int = _abi.TF17_C1
    use_disk: bool = True
    use_halo: bool = True
    periodic: Optional[tuple] = None

    def desc(self) -> "_abi.TF17Desc":
        """The reference's state after TF17Field(disk, halo) and the switches
        (crp_tf17_defaults)."""
        d = _abi.TF17Desc()
        _abi.check(_abi.load().crp_tf17_defaults(int(self.disk), int(self.halo), C.byref(d)))
        d.use_disk, d.use_halo = int(bool(self.use_disk)), int(bool(self.use_halo))
        return d


@dataclass
class SingleModeField:
    """PolarizedSingleModeMagneticField(B_0, wavelength, sigma, r_0, e_1, e_2,
    flagAmplitudeRms, flagPolarizationHelicity, flagMode)
    (PolarizedSingleModeMagneticField.cpp:5): one polarised mode, SI units;
    the flags as strings, as the reference takes them."""
    b0: float
    wavelength: float
    sigma: float
    r0: Sequence[float] = (0.0, 0.0, 0.0)
    e1: Sequence[float] = (1.0, 0.0, 0.0)
    e2: Sequence[float] = (0.0, 1.0, 0.0)
    amplitude_rms: str = "amplitude"
    polarization_helicity: str = "polarization"
    mode: str = "elliptical"
    periodic: Optional[tuple] = None

    def desc(self) -> "_abi.SingleModeDesc":
        """The constructor's checks and derived values (crp_single_mode_field)."""
        flags = ({"amplitude": 0, "rms": 1}.get(self.amplitude_rms, -1),
                 {"polarization": 0, "helicity": 1}.get(self.polarization_helicity, -1),
                 {"elliptical": 0, "circular": 1, "linear": 2}.get(self.mode, -1))
        d = _abi.SingleModeDesc()
        v = [(C.c_double * 3)(*map(float, a)) for a in (self.r0, self.e1, self.e2)]
        _abi.check(_abi.load().crp_single_mode_field(float(self.b0), float(self.wavelength), float(self.sigma),
                                                     v[0], v[1], v[2], *flags, C.byref(d)))
        return d


@dataclass
class KST24Field:
    """KST24Field() (KST24Field.cpp:15): the galactic field of Korochkin,
    Semikoz & Tinyakov 2024 -- toroidal halo, X field, Local Bubble shell and
    five logarithmic spiral arms; no parameters."""
    periodic: Optional[tuple] = None

    @staticmethod
    def desc() -> "_abi.KST24Desc":
        """The constructor's parameters (crp_kst24_defaults)."""
        d = _abi.KST24Desc()
        _abi.check(_abi.load().crp_kst24_defaults(C.byref(d)))
        return d


@dataclass
class CMZField:
    """CMZField() (CMZField.cpp:6), the Galactic-centre field of Guenduez et
    al., with its switches (setUseMCField, setUseICField, setUseNTFField,
    setUseRadioArc): molecular clouds, the intercloud medium (on by default),
    non-thermal filaments and the radio arc."""
    use_mc: bool = False
    use_ic: bool = True
    use_ntf: bool = False
    use_radio_arc: bool = False
    periodic: Optional[tuple] = None

    def desc(self) -> "_abi.CMZDesc":
        """The objects of the four parts (crp_cmz_defaults) with these switches."""
        d = _abi.CMZDesc()
        _abi.check(_abi.load().crp_cmz_defaults(C.byref(d)))
        d.use_mc, d.use_ic = int(bool(self.use_mc)), int(bool(self.use_ic))
        d.use_ntf, d.use_radio_arc = int(bool(self.use_ntf)), int(bool(self.use_radio_arc))
        return d


@dataclass
class ArchimedeanSpiralField:
    """ArchimedeanSpiralField(B_0, R_0, Omega, V_w) (ArchimedeanSpiralField.cpp:5):
    a radial field b0 (r0 / r)^2 wound into an Archimedean spiral by the
    rotation omega over the wind speed vw, reversed below z = 0 (SI units)."""
    b0: float
    r0: float
    omega: float
    vw: float
    periodic: Optional[tuple] = None


def jf12_random_striated(seed: int) -> ScalarGrid:
    """JF12Field::randomStriated(seed) (JF12Field.cpp:86): a periodic 100^3
    Grid1f at the origin with 0.1 kpc spacing, each cell round(rand()) * 2 - 1
    from crpropa::Random seeded with seed (which must not be 0: the reference
    then seeds from the system's entropy)."""
    from . import units as U
    if seed == 0:
        raise ValueError("seed 0 is not reproducible")
    n = 100
    draws = np.empty(n ** 3, np.float64)
    _abi.check(_abi.load().crp_random_draws(int(seed), 0, n ** 3, 0.0, 0.0, 0.0,
                                            draws.ctypes.data_as(C.POINTER(C.c_double))))
    v = (np.floor(draws + 0.5) * 2 - 1).astype(np.float32).reshape(n, n, n)
    return ScalarGrid(v, (0.0, 0.0, 0.0), (0.1 * U.kpc,) * 3, reflective=False)


@dataclass
class PlaneWaveField:
    """PlaneWaveTurbulence modes (PlaneWaveTurbulence.cpp:79)."""
    xi: np.ndarray
    kappa: np.ndarray
    k: np.ndarray
    beta: np.ndarray
    ak: np.ndarray
    spectrum: tuple = (0.0, 1.0, 1.0, 1.0, 5.0 / 3.0, 4.0)  # brms lmin lmax lbendover s q
    seed: int = 0
    periodic: Optional[tuple] = None


@dataclass
class UniformField:
    value: Sequence[float]
    periodic: Optional[tuple] = None


@dataclass
class ToroidalField:
    """B = b0 (-y, x, 0) / sqrt(x^2 + y^2)."""
    b0: float
    periodic: Optional[tuple] = None


@dataclass
class Propagation:
    propagator: int               # _abi.PROP_CK / PROP_BP / PROP_SDE
    tolerance: float
    min_step: float
    max_step: float
    epsilon: float = 0.1
    alpha: float = 1.0 / 3.0
    scale: float = 1.0
    # DiffusionSDE's advection field (DiffusionSDE(magneticField, advectionField, ...),
    # DiffusionSDE.cpp:34): up to four of the classes below, summed in order
    advection: Sequence = ()


def _adv(kind, **kw) -> "_abi.AdvectionDesc":
    d = _abi.AdvectionDesc()
    d.kind = kind
    for k, v in kw.items():
        if k in ("value", "origin"):
            for a in range(3):
                getattr(d, k)[a] = float(v[a])
        else:
            setattr(d, k, int(v) if k == "cool_upstream" else float(v))
    return d


@dataclass
class UniformAdvectionField:
    """UniformAdvectionField(value) (AdvectionField.cpp:29) [m/s]."""
    value: Sequence[float]

    def desc(self):
        return _adv(_abi.ADVECTION_UNIFORM, value=self.value)


@dataclass
class ConstantSphericalAdvectionField:
    """ConstantSphericalAdvectionField(origin, vWind) (AdvectionField.cpp:49)."""
    origin: Sequence[float]
    v_wind: float

    def desc(self):
        return _adv(_abi.ADVECTION_CONSTANT_SPHERICAL, origin=self.origin, v=self.v_wind)


@dataclass
class SphericalAdvectionField:
    """SphericalAdvectionField(origin, radius, vMax, tau, alpha) (AdvectionField.cpp:93)."""
    origin: Sequence[float]
    radius: float
    v_max: float
    tau: float
    alpha: float

    def desc(self):
        return _adv(_abi.ADVECTION_SPHERICAL, origin=self.origin, radius=self.radius, v=self.v_max,
                    tau=self.tau, alpha=self.alpha)


@dataclass
class OneDimensionalCartesianShock:
    """OneDimensionalCartesianShock(compressionRatio, vUp, lShock) (AdvectionField.cpp:182)."""
    compression: float
    v_up: float
    l_shock: float

    def desc(self):
        return _adv(_abi.ADVECTION_CARTESIAN_SHOCK, compression=self.compression, v=self.v_up,
                    length=self.l_shock)


@dataclass
class OneDimensionalSphericalShock:
    """OneDimensionalSphericalShock(rShock, vUp, compressionRatio, lShock,
    coolUpstream) (AdvectionField.cpp:246)."""
    r_shock: float
    v_up: float
    compression: float
    l_shock: float
    cool_upstream: bool

    def desc(self):
        return _adv(_abi.ADVECTION_SPHERICAL_SHOCK_1D, radius=self.r_shock, v=self.v_up,
                    compression=self.compression, length=self.l_shock, cool_upstream=self.cool_upstream)


@dataclass
class ObliqueAdvectionShock:
    """ObliqueAdvectionShock(compressionRatio, vXUp, vY, lShock) (AdvectionField.cpp:353)."""
    compression: float
    v_x_up: float
    v_y: float
    l_shock: float

    def desc(self):
        return _adv(_abi.ADVECTION_OBLIQUE_SHOCK, compression=self.compression, v=self.v_x_up, vy=self.v_y,
                    length=self.l_shock)


@dataclass
class OneDimensionalTimeDependentShock:
    """OneDimensionalTimeDependentShock(v_sh, v1, v0, l_sh)
    (TimeDependentAdvectionField.cpp:7) with setShockPosition (x_sh0, default
    0) and setShockTime (t_sh0, default 0): depends on the candidate's time."""
    v_sh: float
    v1: float
    v0: float
    l_sh: float
    x_sh0: float = 0.0
    t_sh0: float = 0.0

    def desc(self):
        return _adv(_abi.ADVECTION_TIME_SHOCK, v=self.v_sh, v1=self.v1, v0=self.v0, length=self.l_sh,
                    x0=self.x_sh0, t0=self.t_sh0)


@dataclass
class SedovTaylorBlastWave:
    """SedovTaylorBlastWave(E0, rho0, l_sh) (TimeDependentAdvectionField.cpp:97):
    depends on the candidate's time."""
    energy: float
    density: float
    l_sh: float

    def desc(self):
        return _adv(_abi.ADVECTION_SEDOV_TAYLOR, energy=self.energy, density=self.density, length=self.l_sh)


@dataclass
class SphericalAdvectionShock:
    """SphericalAdvectionShock(origin, r_0, v_0, lambda) (AdvectionField.cpp:432)
    with setRRot (default r_0) and setAzimuthalSpeed (default 0)."""
    origin: Sequence[float]
    r_0: float
    v_0: float
    lambda_: float
    r_rot: Optional[float] = None
    v_phi: float = 0.0

    def desc(self):
        return _adv(_abi.ADVECTION_SPHERICAL_SHOCK, origin=self.origin, radius=self.r_0, v=self.v_0,
                    length=self.lambda_, r_rot=self.r_0 if self.r_rot is None else self.r_rot, v_phi=self.v_phi)


@dataclass
class MaxTrajectoryLength:
    max_length: float = 0.0
    per_candidate: bool = False
    record: bool = False


@dataclass
class Feature:
    """One observer feature (crp_observer_feature_desc): a, b, r, step and
    particle_id as the feature kind uses them."""
    kind: int
    a: Sequence[float] = (0.0, 0.0, 0.0)
    b: Sequence[float] = (0.0, 0.0, 0.0)
    r: float = 0.0
    step: float = 0.0
    particle_id: int = 0


@dataclass
class ObserverSpec:
    """Observer (Observer.cpp:27): the single sphere/detect-all feature given
    by feature/center/radius, or the list `features` (at most 4)."""
    feature: int = _abi.OBSERVER_SURFACE_SPHERE
    center: Sequence[float] = (0.0, 0.0, 0.0)
    radius: float = 0.0
    deactivate: bool = True
    record: bool = False
    features: Optional[List[Feature]] = None


@dataclass
class BoundarySpec:
    """Spherical/Cubic/Ellipsoidal/CylindricalBoundary (Boundary.cpp:171-303):
    a = centre / origin / first focal point, b = second focal point, size =
    radius / edge / major axis / height, radius = cylinder radius."""
    kind: int
    a: Sequence[float] = (0.0, 0.0, 0.0)
    b: Sequence[float] = (0.0, 0.0, 0.0)
    size: float = 0.0
    radius: float = 0.0
    margin: float = 0.1 * 3.0856775814913673e19  # 0.1 kpc, the reference default
    limit_step: bool = True
    record: bool = False


@dataclass
class ChainSpec:
    fields: List[object]
    modules: List[object]
    precision: int = _abi.PRECISION_FP64
    seed: int = 0
    _keep: list = field(default_factory=list, repr=False)

    def __getstate__(self):
        # the ctypes views of the last desc() are not picklable; desc()
        # rebuilds them
        state = dict(self.__dict__)
        state["_keep"] = []
        return state

    def desc(self) -> _abi.PlanDesc:
        self._keep = []
        comps = (_abi.FieldComponent * max(1, len(self.fields)))()
        for i, f in enumerate(self.fields):
            self._fill_component(comps[i], f)
        mods = (_abi.ModuleDesc * len(self.modules))()
        for i, m in enumerate(self.modules):
            self._fill_module(mods[i], m)
        self._keep += [comps, mods]
        d = _abi.PlanDesc()
        d.abi_version = _abi.ABI_VERSION
        d.precision = int(self.precision)
        d.fields = C.cast(comps, C.POINTER(_abi.FieldComponent))
        d.n_fields = len(self.fields)
        d.n_modules = len(self.modules)
        d.modules = C.cast(mods, C.POINTER(_abi.ModuleDesc))
        d.seed = int(self.seed)
        self._keep.append(d)
        return d

    def _arr(self, a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype)
        self._keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_float if dtype == np.float32 else C.c_double))

    def _fill_component(self, c, f):
        per = getattr(f, "periodic", None)
        if per is not None:
            o, e, refl = per
            c.periodic = 1
            c.periodic_origin[:] = _v3(o)
            c.periodic_extends[:] = _v3(e)
            c.periodic_reflective = int(bool(refl))
        if isinstance(f, GridField):
            c.kind = _abi.FIELD_GRID
            self._fill_grid(c.grid, f, 3)
        elif isinstance(f, ModulatedGridField):
            c.kind = _abi.FIELD_MODULATED_GRID
            self._fill_grid(c.grid, f.grid, 3)
            self._fill_grid(c.modulation, f.modulation, 1)
        elif isinstance(f, JF12Field):
            c.kind = _abi.FIELD_JF12
            c.jf12 = f.parameters()
            j = c.jf12
            j.use_regular, j.use_disk = int(bool(f.use_regular)), int(bool(f.use_disk))
            j.use_toroidal_halo, j.use_x = int(bool(f.use_toroidal_halo)), int(bool(f.use_x))
            j.use_striated = int(bool(f.striated is not None if f.use_striated is None else f.use_striated))
            j.use_turbulent = int(bool(f.turbulent is not None if f.use_turbulent is None else f.use_turbulent))
            if f.striated is not None:
                self._fill_grid(c.modulation, f.striated, 1)
            if f.turbulent is not None:
                self._fill_grid(c.grid, f.turbulent, 3)
        elif isinstance(f, UF23Field):
            c.kind = _abi.FIELD_UF23
            c.uf23 = UF23Field.defaults(f.model)
        elif isinstance(f, PT11Field):
            c.kind = _abi.FIELD_PT11
            c.pt11 = f.desc()
        elif isinstance(f, TF17Field):
            c.kind = _abi.FIELD_TF17
            c.tf17 = f.desc()
        elif isinstance(f, SingleModeField):
            c.kind = _abi.FIELD_SINGLE_MODE
            c.single_mode = f.desc()
        elif isinstance(f, KST24Field):
            c.kind = _abi.FIELD_KST24
            c.kst24 = f.desc()
        elif isinstance(f, CMZField):
            c.kind = _abi.FIELD_CMZ
            c.cmz = f.desc()
        elif isinstance(f, ArchimedeanSpiralField):
            c.kind = _abi.FIELD_ARCHIMEDEAN_SPIRAL
            c.archimedean.b0, c.archimedean.r0 = float(f.b0), float(f.r0)
            c.archimedean.omega, c.archimedean.vw = float(f.omega), float(f.vw)
        elif isinstance(f, PlaneWaveField):
            c.kind = _abi.FIELD_PLANE_WAVE
            w = c.plane_wave
            w.n_modes = len(f.k)
            w.seed = int(f.seed)
            w.xi = self._arr(f.xi, np.float64)
            w.kappa = self._arr(f.kappa, np.float64)
            w.k = self._arr(f.k, np.float64)
            w.beta = self._arr(f.beta, np.float64)
            w.ak = self._arr(f.ak, np.float64)
            w.brms, w.lmin, w.lmax, w.lbendover, w.sindex, w.qindex = f.spectrum
        elif isinstance(f, UniformField):
            c.kind = _abi.FIELD_UNIFORM
            c.uniform[:] = _v3(f.value)
        elif isinstance(f, ToroidalField):
            c.kind = _abi.FIELD_TOROIDAL
            c.toroidal_b0 = float(f.b0)
        else:
            raise TypeError(f"unsupported field component {type(f).__name__}")

    def _fill_grid(self, g, f, comps):
        v = np.ascontiguousarray(f.values, dtype=np.float32)
        if comps == 3 and (v.ndim != 4 or v.shape[3] != 3):
            raise ValueError("grid values must have shape (nx, ny, nz, 3)")
        if comps == 1 and v.ndim != 3:
            raise ValueError("scalar grid values must have shape (nx, ny, nz)")
        g.values = self._arr(v, np.float32)
        g.nx, g.ny, g.nz = v.shape[:3]
        g.origin[:] = _v3(f.origin)
        g.spacing[:] = _v3(f.spacing)
        g.reflective = int(bool(f.reflective))
        g.clip_volume = int(bool(f.clip_volume))
        g.interpolation = int(f.interpolation)

    @staticmethod
    def _fill_module(d, m):
        if isinstance(m, Propagation):
            d.kind = _abi.MODULE_PROPAGATION
            d.propagator = int(m.propagator)
            d.tolerance, d.min_step, d.max_step = float(m.tolerance), float(m.min_step), float(m.max_step)
            d.sde_epsilon, d.sde_alpha, d.sde_scale = float(m.epsilon), float(m.alpha), float(m.scale)
            adv = list(m.advection or ())
            if len(adv) > _abi.MAX_ADVECTION:
                raise ValueError(f"DiffusionSDE: at most {_abi.MAX_ADVECTION} advection fields")
            d.n_advection = len(adv)
            for i, a in enumerate(adv):
                d.advection[i] = a.desc()
        elif isinstance(m, MaxTrajectoryLength):
            d.kind = _abi.MODULE_MAX_TRAJECTORY_LENGTH
            d.max_length = float(m.max_length)
            d.per_candidate_length = int(bool(m.per_candidate))
            d.record = int(bool(m.record))
        elif isinstance(m, ObserverSpec):
            d.kind = _abi.MODULE_OBSERVER
            d.observer_feature = int(m.feature)
            d.sphere_center[:] = _v3(m.center)
            d.sphere_radius = float(m.radius)
            d.deactivate_on_detection = int(bool(m.deactivate))
            d.record = int(bool(m.record))
            feats = m.features or []
            if len(feats) > _abi.MAX_OBSERVER_FEATURES:
                raise ValueError(f"at most {_abi.MAX_OBSERVER_FEATURES} observer features")
            d.n_features = len(feats)
            for i, f in enumerate(feats):
                fd = d.features[i]
                fd.kind, fd.particle_id = int(f.kind), int(f.particle_id)
                fd.a[:], fd.b[:] = _v3(f.a), _v3(f.b)
                fd.r, fd.step = float(f.r), float(f.step)
        elif isinstance(m, BoundarySpec):
            d.kind = _abi.MODULE_BOUNDARY
            d.boundary = int(m.kind)
            d.boundary_a[:], d.boundary_b[:] = _v3(m.a), _v3(m.b)
            d.boundary_size, d.boundary_radius = float(m.size), float(m.radius)
            d.boundary_margin = float(m.margin)
            d.boundary_limit_step = int(bool(m.limit_step))
            d.record = int(bool(m.record))
        else:
            raise TypeError(f"unsupported module {type(m).__name__}")
