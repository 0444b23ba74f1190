/*
 * crp_gpu.h -- C-ABI of the B200 charged-particle stepping engine.
 *
 * This is the drop-in boundary for CRPropa's charged-particle stepping path:
 * a chain of one propagation module (PropagationCK, PropagationBP or
 * DiffusionSDE) over a magnetic field (MagneticFieldGrid over a Grid3f,
 * ModulatedMagneticFieldGrid, PeriodicMagneticField, PlaneWaveTurbulence,
 * UniformMagneticField, JF12Field, UF23Field, PT11Field, ArchimedeanSpiralField, TF17Field,
 * PolarizedSingleModeMagneticField, a
 * MagneticFieldList of those,
 * or a toroidal field), followed by MaximumTrajectoryLength, Observer and
 * boundary modules, run to completion over a set of candidates.  It replaces, for such chains,
 *
 *   ModuleList::run(const candidate_vector_t*, bool, bool)
 *       include/crpropa/ModuleList.h:43, src/ModuleList.cpp.in:97
 *   ModuleList::run(SourceInterface*, size_t, bool, bool)
 *       include/crpropa/ModuleList.h:44, src/ModuleList.cpp.in:153
 *
 * Only plain C types cross this boundary: pointers, sizes and POD structs.
 * No call throws; every entry point returns a crp_status and leaves a
 * message retrievable with crp_last_error().  A C++ wrapper maps a non-zero
 * status to std::runtime_error, which SWIG maps to a Python RuntimeError
 * (python/1_swig.i:53-63 of the reference).
 *
 * Units are SI throughout, as in include/crpropa/Units.h: metres, seconds,
 * joules, coulombs, tesla.
 */
#ifndef CRP_GPU_H
#define CRP_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CRP_ABI_VERSION 9u

typedef enum crp_status {
    CRP_OK = 0,
    CRP_ERR_INVALID_ARGUMENT = 1, /* a parameter the reference setters would reject */
    CRP_ERR_UNSUPPORTED = 2,      /* chain or field outside the device path: run the CPU ModuleList */
    CRP_ERR_CUDA = 3,             /* a CUDA runtime call failed */
    CRP_ERR_OUT_OF_MEMORY = 4,
    CRP_ERR_TIMEOUT = 5,          /* a bounded device-side wait ran out */
    CRP_ERR_CANCELLED = 6,        /* the host cancel flag was raised */
    CRP_ERR_CAPACITY = 7,         /* a size beyond a documented limit */
    CRP_ERR_NO_DEVICE = 8         /* no CUDA device is visible */
} crp_status;

/* ------------------------------------------------------------------------
 * Magnetic field description
 * ---------------------------------------------------------------------- */

enum crp_field_kind {
    CRP_FIELD_GRID = 1,       /* MagneticFieldGrid over Grid3f (MagneticFieldGrid.cpp:17) */
    CRP_FIELD_PLANE_WAVE = 2, /* PlaneWaveTurbulence (PlaneWaveTurbulence.cpp:231) */
    CRP_FIELD_UNIFORM = 3,    /* UniformMagneticField (MagneticField.h:109) */
    CRP_FIELD_TOROIDAL = 4,   /* B = b0 * (-y, x, 0) / r, r = sqrt(x^2 + y^2) */
    CRP_FIELD_MODULATED_GRID = 5, /* ModulatedMagneticFieldGrid: Grid3f times a Grid1f
                                     modulation (MagneticFieldGrid.cpp:51) */
    CRP_FIELD_JF12 = 6,           /* JF12Field / PlanckJF12bField (JF12Field.cpp:8-376) */
    CRP_FIELD_UF23 = 7,           /* UF23Field (UF23Field.cpp:59-558) */
    CRP_FIELD_PT11 = 8,           /* PT11Field (PT11Field.cpp:8-130) */
    CRP_FIELD_ARCHIMEDEAN_SPIRAL = 9, /* ArchimedeanSpiralField (ArchimedeanSpiralField.cpp:5-49) */
    CRP_FIELD_TF17 = 10,          /* TF17Field (TF17Field.cpp:10-307) */
    CRP_FIELD_SINGLE_MODE = 11,   /* PolarizedSingleModeMagneticField
                                     (PolarizedSingleModeMagneticField.cpp:5-64) */
    CRP_FIELD_KST24 = 12,         /* KST24Field (KST24Field.cpp:15-374) */
    CRP_FIELD_CMZ = 13            /* CMZField (CMZField.cpp:6-304) */
};

/* UF23Field::ModelType (UF23Field.h), same order. */
enum crp_uf23_model {
    CRP_UF23_BASE = 0,
    CRP_UF23_NECL = 1,
    CRP_UF23_EXPX = 2,
    CRP_UF23_SPUR = 3,
    CRP_UF23_CRE10 = 4,
    CRP_UF23_SYNCG = 5,
    CRP_UF23_TWISTX = 6,
    CRP_UF23_NEBCOR = 7
};

/* Grid::setInterpolationType (Grid.h:255; enum interpolationType, Grid.h:24). */
enum crp_interpolation {
    CRP_INTERPOLATION_TRILINEAR = 0,        /* Grid.h:539 */
    CRP_INTERPOLATION_TRICUBIC = 1,         /* Grid.h:459 (Vector3f: the SIMD form), Grid.h:504 */
    CRP_INTERPOLATION_NEAREST_NEIGHBOUR = 2 /* closestValue, Grid.h:383 */
};

/* Grid3f payload and GridProperties (Grid.h:75).  values holds Nx*Ny*Nz
 * Vector3f cells (12 bytes each, x y z floats), cell (ix,iy,iz) at
 * ix*Ny*Nz + iy*Nz + iz (Grid.h:338).  Host memory. */
typedef struct crp_grid3f_desc {
    const float *values;
    uint64_t nx, ny, nz;
    double origin[3];  /* lower-left-front corner of the volume */
    double spacing[3];
    int32_t reflective;  /* Grid::setReflective */
    int32_t clip_volume; /* Grid::setClipVolume */
    int32_t interpolation; /* crp_interpolation */
    int32_t _pad;
} crp_grid3f_desc;

/* Wave modes of a PlaneWaveTurbulence (PlaneWaveTurbulence.cpp:79-229),
 * as produced by crp_plane_wave_modes().  Host memory. */
typedef struct crp_plane_wave_desc {
    int32_t n_modes;
    int32_t seed;        /* constructor seed the modes were drawn with */
    const double *xi;    /* 3*n_modes, polarisation unit vectors, mode-major */
    const double *kappa; /* 3*n_modes, propagation unit vectors, mode-major */
    const double *k;     /* n_modes, wave numbers [1/m] */
    const double *beta;  /* n_modes, phases */
    const double *ak;    /* n_modes, amplitudes [T] */
    /* TurbulenceSpectrum the modes came from (TurbulentField.h:17): the
     * device reads only the mode arrays above. */
    double brms, lmin, lmax, lbendover, sindex, qindex;
} crp_plane_wave_desc;

/* Constructor a crp_jf12_desc's parameters come from. */
enum crp_jf12_variant {
    CRP_JF12_JF12 = 0,       /* JF12Field (JF12Field.cpp:8) */
    CRP_JF12_PLANCK = 1,     /* PlanckJF12bField (JF12Field.cpp:352) */
    CRP_JF12_SOLENOIDAL = 2  /* JF12FieldSolenoidal (JF12FieldSolenoidal.cpp:8) */
};

/* Parameters of the Jansson-Farrar 2012 galactic field as JF12Field holds
 * them (JF12Field.h, set by the constructors JF12Field.cpp:8 and :352), SI
 * units, and the state JF12FieldSolenoidal adds (JF12FieldSolenoidal.h:35-55).
 * crp_jf12_defaults() and crp_jf12_solenoidal() fill them.  The striated grid
 * (a Grid1f, one float per cell, read by nearest value, JF12Field.cpp:296) is
 * the component's `modulation` grid and the turbulent grid (a Grid3f,
 * JF12Field.cpp:340) its `grid`. */
typedef struct crp_jf12_desc {
    int32_t use_regular, use_disk, use_toroidal_halo, use_x, use_striated, use_turbulent;
    int32_t variant;                    /* constructor the parameters come from: 0 JF12Field,
                                           1 PlanckJF12bField */
    int32_t _pad;
    double kpc;                         /* the kiloparsec the model's constants are written in */
    double sin_pitch, cos_pitch, tan90_minus_pitch;
    double r_arms[8];
    double b_ring, h_disk, w_disk;
    double b_disk[8];
    double b_north, b_south, r_north, r_south, w_halo, z0;
    double b_x, sin_theta_x0, cos_theta_x0, tan_theta_x0, r_xc, r_x;
    double sqrt_beta;                   /* striation */
    double b_disk_turb[8];
    double b_disk_turb5, z_disk_turb, b_halo_turb, r_halo_turb, z_halo_turb;
    /* JF12FieldSolenoidal only (variant CRP_JF12_SOLENOIDAL): */
    double cot_pitch, cot_theta_x0;     /* 1 / tan of the pitch and of thetaX0 */
    double z_s;                         /* X field: parabolic field lines below |z| = z_s */
    double delta;                       /* the transition width the constructor was given */
    double r1, r2, r1s, r2s;            /* disk between r1 and r2, transitions [r1, r1s] and [r2s, r2] */
    double phi0_arms[11];               /* azimuths where the arms cross r1, periodically closed */
    double b_arms[11];                  /* arm strengths at r1, periodically closed (bDisk) */
    double phi_coeff[10];               /* the azimuth integral H(phi) = phi_coeff[j] + b_arms[j] phi */
} crp_jf12_desc;

/* Parameters of a UF23Field model (UF23Field.h, UF23Field::EPar order; set by
 * the constructor, UF23Field.cpp:59-266) in the model's own units: kpc,
 * microgauss, radians, Myr.  crp_uf23_defaults() fills them. */
typedef struct crp_uf23_desc {
    int32_t model; /* crp_uf23_model */
    int32_t _pad;
    double disk_b1, disk_b2, disk_b3, disk_h, disk_phase1, disk_phase2, disk_phase3, disk_pitch, disk_w;
    double poloidal_a, poloidal_b, poloidal_p, poloidal_r, poloidal_w, poloidal_z, poloidal_xi;
    double spur_center, spur_length, spur_width, striation;
    double toroidal_bn, toroidal_bs, toroidal_r, toroidal_w, toroidal_z, twisting_time;
    double sin_pitch, cos_pitch, tan_pitch; /* of disk_pitch */
    double max_radius_squared;              /* kpc^2; B = 0 beyond */
    double kpc;                             /* position unit [m] */
    double microgauss;                      /* field unit [T] */
} crp_uf23_desc;

/* State of a PT11Field (PT11Field.h:26-46), SI units: the ASS/BSS disk and
 * halo switches and the parameters the constructor and the setters set
 * (PT11Field.cpp:8-64), with SetParams' derived values (PT11Field.cpp:28).
 * crp_pt11_defaults() and crp_pt11_use() fill it. */
typedef struct crp_pt11_desc {
    int32_t use_ass, use_bss, use_halo, _pad;
    double d, r_sun, r_c, z0_d, b0_d;                     /* disk [m], [T] */
    double z0_h, r0_h, b0_hn, b0_hs, z11_h, z12_h;        /* halo [m], [T] */
    double pitch, cos_pitch, sin_pitch, phi, cos_phi;     /* pitch [rad] and SetParams' values */
} crp_pt11_desc;

/* ArchimedeanSpiralField(B_0, R_0, Omega, V_w) (ArchimedeanSpiralField.h:46), SI units. */
typedef struct crp_archimedean_desc {
    double b0;    /* radial field strength at r0 [T] */
    double r0;    /* reference radius [m] */
    double omega; /* angular velocity of the rotation [1/s] */
    double vw;    /* asymptotic wind speed [m/s] */
} crp_archimedean_desc;

/* TF17DiskModel and TF17HaloModel (TF17Field.h:20-21), same order. */
enum crp_tf17_disk { CRP_TF17_AD1 = 0, CRP_TF17_BD1 = 1, CRP_TF17_DD1 = 2 };
enum crp_tf17_halo { CRP_TF17_C0 = 0, CRP_TF17_C1 = 1 };

/* State of a TF17Field (TF17Field.h:27-57), SI units: the disk and halo
 * models and switches and the parameters TF17Field(disk, halo) sets
 * (TF17Field.cpp:10-118), cot_p0 as set_p0 forms it (TF17Field.cpp:146).
 * Parameters a model combination does not set are 0 here (the reference
 * leaves them uninitialised; that model never reads them).
 * crp_tf17_defaults() fills it. */
typedef struct crp_tf17_desc {
    int32_t disk_model, halo_model;                  /* crp_tf17_disk, crp_tf17_halo */
    int32_t use_disk, use_halo;                      /* setUseDiskField, setUseHaloField */
    double a_disk, z1_disk, r1_disk, b1_disk, l_disk, phi_star_disk, h_disk;
    double a_halo, z1_halo, b1_halo, l_halo, phi_star_halo;
    double p0, cot_p0, h_p, l_p;
    double epsilon;                                  /* numeric_limits<double>::epsilon() */
} crp_tf17_desc;

/* PolarizedSingleModeMagneticField's derived state (PolarizedSingleModeMagneticField.h:34-38),
 * SI units: B = b_max (u1 cos(k . (x - r0)) + u2 sigma sin(k . (x - r0))).
 * crp_single_mode_field() forms it from the constructor's arguments. */
typedef struct crp_single_mode_desc {
    double b_max, sigma;
    double r0[3];
    double u1[3], u2[3]; /* unit vectors of e_1 and e_2 */
    double k[3];         /* wave vector, along e_2 x e_1, |k| = 2 pi / wavelength */
    /* the constructor's own arguments (the device reads the values above) */
    double b0, wavelength;
    double e1[3], e2[3];
    int32_t amplitude_rms, polarization_helicity, mode, _pad;
} crp_single_mode_desc;

/* The constructor's string flags as numbers. */
enum crp_single_mode_flag {
    CRP_SINGLE_MODE_AMPLITUDE = 0, CRP_SINGLE_MODE_RMS = 1,             /* flagAmplitudeRms */
    CRP_SINGLE_MODE_POLARIZATION = 0, CRP_SINGLE_MODE_HELICITY = 1,     /* flagPolarizationHelicity */
    CRP_SINGLE_MODE_ELLIPTICAL = 0, CRP_SINGLE_MODE_CIRCULAR = 1, CRP_SINGLE_MODE_LINEAR = 2 /* flagMode */
};

/* One logarithmic spiral arm of KST24Field (KST24Field.h:53-120), the
 * model's units: strength [gauss], pitch, phase and the cross-section's
 * growth [degrees], centre shift, cross-section radii (height, plane) and the
 * ranges in r and z [kpc], the cross-section's super-ellipse exponent. */
typedef struct crp_kst24_arm {
    double b, pitch_deg, phi0_deg, x_shift, y_shift, arc_radius1, arc_radius2, arc_eps, arc_div_deg;
    double rmin, rmax, zmin, zmax;
} crp_kst24_arm;

/* KST24Field's parameters (KST24Field.h:22-120, set by the constructor,
 * KST24Field.cpp:15-124) in the model's units (kpc, gauss).
 * crp_kst24_defaults() fills them. */
typedef struct crp_kst24_desc {
    double north_b, north_zmin, north_zmax, north_rmin, north_rmax; /* toroidal halo, north */
    double south_b, south_zmin, south_zmax, south_rmin, south_rmax; /* and south */
    double x_b, x_rmin, x_rmax, x_theta_rad;                        /* X field */
    double lb_b, lb_rmin, lb_dr, lb_x0, lb_y0, lb_z0;               /* Local Bubble shell */
    double lb_dir[3];                                               /* its field direction */
    crp_kst24_arm arms[5]; /* Scutum, Carina-Sagittarius, Local, Perseus 1, Perseus 2 */
    double kpc, gauss;     /* the units [m], [T] */
} crp_kst24_desc;

/* A molecular cloud of CMZField's azimuthal model (CMZField::BAz,
 * CMZField.cpp:36): centre [m], strength B1 [gauss], eta, radius R [m]. */
typedef struct crp_cmz_cloud { double mid[3], b1, eta, r; } crp_cmz_cloud;

/* An object of CMZField's poloidal model (CMZField::BPol, CMZField.cpp:18):
 * centre [m], strength (B1 / eta) and the model parameters a [1/m^2] and L [m]. */
typedef struct crp_cmz_poloidal { double mid[3], b, a, l; } crp_cmz_poloidal;

/* CMZField (CMZField.h:21-79), the Galactic-centre field of Guenduez et al.:
 * the switches (setUseMCField, setUseICField, setUseNTFField, setUseRadioArc)
 * and the objects getMCField, getICField, getNTFField and getRadioArcField
 * sum, in their order (CMZField.cpp:116-287).  crp_cmz_defaults() fills it. */
typedef struct crp_cmz_desc {
    int32_t use_mc, use_ic, use_ntf, use_radio_arc;
    crp_cmz_cloud clouds[12];     /* molecular clouds */
    double sgra_shift[3];         /* Sgr A*: added to the position */
    double sgra_r, sgra_b1;       /* its radius [m] and strength */
    crp_cmz_poloidal ic;          /* the intercloud medium [T] */
    crp_cmz_poloidal ntf[7];      /* non-thermal filaments; the last (the Pelican) with y and z swapped */
    crp_cmz_poloidal radio_arc;
    double gauss;                 /* [T] */
} crp_cmz_desc;

/* crp_pt11_use() switches, PT11Field::setUseASS / setUseBSS / setUseHalo. */
enum crp_pt11_switch { CRP_PT11_ASS = 0, CRP_PT11_BSS = 1, CRP_PT11_HALO = 2 };

/* One summand of the field (a MagneticFieldList of these is their sum,
 * MagneticField.cpp:64).  A component may be wrapped in a
 * PeriodicMagneticField (MagneticField.cpp:41). */
typedef struct crp_field_component {
    int32_t kind;
    int32_t periodic;            /* wrap in PeriodicMagneticField */
    int32_t periodic_reflective; /* PeriodicMagneticField reflective flag */
    int32_t _pad0;
    double periodic_origin[3];
    double periodic_extends[3];
    crp_grid3f_desc grid;
    crp_plane_wave_desc plane_wave;
    double uniform[3];
    double toroidal_b0;
    /* CRP_FIELD_MODULATED_GRID: the Grid1f modulation, one float per cell
     * (values: nx*ny*nz floats in the same order as a Grid3f's cells);
     * CRP_FIELD_JF12: the striated grid */
    crp_grid3f_desc modulation;
    crp_jf12_desc jf12;
    crp_uf23_desc uf23;
    crp_pt11_desc pt11;
    crp_archimedean_desc archimedean;
    crp_tf17_desc tf17;
    crp_single_mode_desc single_mode;
    crp_kst24_desc kst24;
    crp_cmz_desc cmz;
} crp_field_component;

/* ------------------------------------------------------------------------
 * Module chain description (ModuleList order)
 * ---------------------------------------------------------------------- */

enum crp_module_kind {
    CRP_MODULE_PROPAGATION = 1,
    CRP_MODULE_MAX_TRAJECTORY_LENGTH = 2, /* MaximumTrajectoryLength (BreakCondition.cpp:42) */
    CRP_MODULE_OBSERVER = 3,              /* Observer (Observer.cpp:27) */
    CRP_MODULE_BOUNDARY = 4               /* SphericalBoundary, CubicBoundary, EllipsoidalBoundary,
                                             CylindricalBoundary (Boundary.cpp:171-320) */
};

enum crp_propagator {
    CRP_PROP_CK = 1,  /* PropagationCK (PropagationCK.cpp:77) */
    CRP_PROP_BP = 2,  /* PropagationBP (PropagationBP.cpp:62) */
    CRP_PROP_SDE = 3  /* DiffusionSDE  (DiffusionSDE.cpp:47) */
};

enum crp_observer_feature {
    CRP_OBSERVER_SURFACE_SPHERE = 1,   /* ObserverSurface(Sphere) (Observer.cpp:394, Geometry.cpp:41) */
    CRP_OBSERVER_DETECT_ALL = 2,       /* ObserverDetectAll (Observer.cpp:93) */
    CRP_OBSERVER_SURFACE_PLANE = 3,    /* ObserverSurface(Plane) (Geometry.cpp:19): a = x0, b = n */
    CRP_OBSERVER_SURFACE_BOX = 4,      /* ObserverSurface(ParaxialBox) (Geometry.cpp:64): a = corner, b = size */
    CRP_OBSERVER_TRACKING = 5,         /* ObserverTracking (Observer.cpp:109): a = centre, r, step */
    CRP_OBSERVER_1D = 6,               /* Observer1D (Observer.cpp:137) */
    CRP_OBSERVER_INACTIVE_VETO = 7,    /* ObserverInactiveVeto (Observer.cpp:174) */
    CRP_OBSERVER_NUCLEUS_VETO = 8,     /* ObserverNucleusVeto (Observer.cpp:185) */
    CRP_OBSERVER_NEUTRINO_VETO = 9,    /* ObserverNeutrinoVeto (Observer.cpp:196) */
    CRP_OBSERVER_PHOTON_VETO = 10,     /* ObserverPhotonVeto (Observer.cpp:208) */
    CRP_OBSERVER_ELECTRON_VETO = 11,   /* ObserverElectronVeto (Observer.cpp:219) */
    CRP_OBSERVER_PARTICLE_ID_VETO = 12 /* ObserverParticleIdVeto (Observer.cpp:234): particle_id */
};

/* One feature of an Observer; the observer detects when a feature detects
 * and none vetoes (Observer.cpp:27-35), every feature limiting the next step
 * as its checkDetection does. */
typedef struct crp_observer_feature_desc {
    int32_t kind;        /* crp_observer_feature */
    int32_t particle_id; /* CRP_OBSERVER_PARTICLE_ID_VETO */
    double a[3];
    double b[3];
    double r;
    double step;
} crp_observer_feature_desc;

#define CRP_MAX_OBSERVER_FEATURES 4

enum crp_boundary_kind {
    CRP_BOUNDARY_SPHERICAL = 1,  /* SphericalBoundary (Boundary.cpp:216): a = centre, size = radius */
    CRP_BOUNDARY_CUBIC = 2,      /* CubicBoundary (Boundary.cpp:171): a = origin, size */
    CRP_BOUNDARY_ELLIPSOIDAL = 3,/* EllipsoidalBoundary (Boundary.cpp:259): a, b = focal points, size = major axis */
    CRP_BOUNDARY_CYLINDRICAL = 4 /* CylindricalBoundary (Boundary.cpp:303): a = origin, size = height, radius */
};

/* Advection fields of DiffusionSDE (AdvectionField.h:23-265, getField of
 * AdvectionField.cpp:12-420), SI units.  The fields each kind reads:
 *   UNIFORM             value
 *   CONSTANT_SPHERICAL  origin, v (vWind)
 *   SPHERICAL           origin, radius, v (vMax), tau, alpha
 *   CARTESIAN_SHOCK     compression, v (vUp), length (lShock)
 *   SPHERICAL_SHOCK_1D  radius (rShock), v (vUp), compression, length (lShock), cool_upstream
 *   OBLIQUE_SHOCK       compression, v (vXUp), vy, length (lShock)
 *   SPHERICAL_SHOCK     origin, radius (r_0), v (v_0), length (lambda), r_rot, v_phi
 *   TIME_SHOCK          v (v_sh), v1, v0, length (l_sh), x0 (x_sh0), t0 (t_sh0)
 *   SEDOV_TAYLOR        energy (E0), density (rho0), length (l_sh)
 * The last two depend on the candidate's time at the step's start
 * (TimeDependentAdvectionField.cpp:16, :103); inside a list they get time 0,
 * as AdvectionFieldList::getField passes none (AdvectionField.cpp:15). */
enum crp_advection_kind {
    CRP_ADVECTION_UNIFORM = 1,            /* UniformAdvectionField */
    CRP_ADVECTION_CONSTANT_SPHERICAL = 2, /* ConstantSphericalAdvectionField */
    CRP_ADVECTION_SPHERICAL = 3,          /* SphericalAdvectionField */
    CRP_ADVECTION_CARTESIAN_SHOCK = 4,    /* OneDimensionalCartesianShock */
    CRP_ADVECTION_SPHERICAL_SHOCK_1D = 5, /* OneDimensionalSphericalShock */
    CRP_ADVECTION_OBLIQUE_SHOCK = 6,      /* ObliqueAdvectionShock */
    CRP_ADVECTION_SPHERICAL_SHOCK = 7,    /* SphericalAdvectionShock */
    CRP_ADVECTION_TIME_SHOCK = 8,         /* OneDimensionalTimeDependentShock */
    CRP_ADVECTION_SEDOV_TAYLOR = 9        /* SedovTaylorBlastWave */
};
#define CRP_MAX_ADVECTION 4

typedef struct crp_advection_desc {
    int32_t kind;          /* crp_advection_kind */
    int32_t cool_upstream; /* OneDimensionalSphericalShock::setCooling */
    double value[3];
    double origin[3];
    double v, radius, tau, alpha, compression, length, vy, r_rot, v_phi;
    double v1, v0, x0, t0, energy, density;
} crp_advection_desc;

typedef struct crp_module_desc {
    int32_t kind;
    /* CRP_MODULE_PROPAGATION */
    int32_t propagator;
    double tolerance;
    double min_step; /* [m] */
    double max_step; /* [m]; min_step == max_step selects the fixed-step branch */
    double sde_epsilon; /* DiffusionSDE::setEpsilon */
    double sde_alpha;   /* DiffusionSDE::setAlpha */
    double sde_scale;   /* DiffusionSDE::setScale */
    /* DiffusionSDE::setAdvectionField: n_advection fields, summed in order
     * (an AdvectionFieldList, AdvectionField.cpp:12); 0: none */
    int32_t n_advection;
    int32_t _pad_adv;
    crp_advection_desc advection[CRP_MAX_ADVECTION];
    /* CRP_MODULE_MAX_TRAJECTORY_LENGTH */
    double max_length;            /* [m] */
    int32_t per_candidate_length; /* use crp_candidates.max_length[i] instead */
    /* CRP_MODULE_OBSERVER */
    int32_t observer_feature;
    double sphere_center[3];
    double sphere_radius;
    int32_t deactivate_on_detection; /* Observer::setDeactivateOnDetection, default 1 */
    int32_t record;                  /* the detection (or rejection) action writes a record */
    /* CRP_MODULE_OBSERVER with several features: n_features > 0 replaces
     * observer_feature and sphere_* above */
    int32_t n_features;
    /* CRP_MODULE_BOUNDARY */
    int32_t boundary;                /* crp_boundary_kind */
    crp_observer_feature_desc features[CRP_MAX_OBSERVER_FEATURES];
    double boundary_a[3];
    double boundary_b[3];
    double boundary_size;
    double boundary_radius;
    double boundary_margin;          /* setMargin, default 0.1 kpc (0 cylindrical) */
    int32_t boundary_limit_step;     /* setLimitStep, default 1 (0 cylindrical) */
    int32_t _pad1;
} crp_module_desc;

enum crp_precision {
    CRP_PRECISION_FP64 = 0,  /* the reference's arithmetic, operation for operation */
    CRP_PRECISION_MIXED = 1  /* FP32 field and stage arithmetic, FP64 accumulation */
};

typedef struct crp_plan_desc {
    uint32_t abi_version; /* CRP_ABI_VERSION */
    int32_t precision;
    const crp_field_component *fields;
    int32_t n_fields;
    int32_t n_modules;
    const crp_module_desc *modules;
    uint64_t seed; /* key of the counter-based random stream (DiffusionSDE) */
} crp_plan_desc;

/* ------------------------------------------------------------------------
 * Candidate state, structure of arrays (Candidate.h:27, ParticleState.h:22)
 * ---------------------------------------------------------------------- */

enum crp_candidate_flags {
    CRP_FLAG_REJECTED = 1u, /* property "Rejected" set by MaximumTrajectoryLength */
    CRP_FLAG_DETECTED = 2u, /* Observer detection */
    CRP_FLAG_NAN = 4u       /* DiffusionSDE deactivated a NaN position (DiffusionSDE.cpp:177) */
};

/* Every array has n entries.  All pointers are host pointers for crp_run()
 * and device pointers for crp_run_device().  max_length may be NULL unless a
 * module sets per_candidate_length. */
typedef struct crp_candidates {
    int32_t *id;        /* PDG id (ParticleState::setId) */
    double *charge;     /* [C] */
    double *energy;     /* [J] */
    double *x, *y, *z;  /* current position [m] */
    double *dx, *dy, *dz; /* current direction (unit vector) */
    double *px, *py, *pz; /* previous position (Candidate::previous) */
    double *trajectory_length; /* [m] */
    double *time;              /* [s] */
    double *current_step;      /* [m] */
    double *next_step;         /* [m] */
    uint8_t *active;
    uint32_t *flags;     /* crp_candidate_flags */
    double *max_length;  /* per-candidate MaximumTrajectoryLength [m], optional */
    uint64_t *step_count; /* accepted steps taken so far, optional */
} crp_candidates;

/* Output records written by an Observer or MaximumTrajectoryLength module
 * with record != 0 (the detection / reject action, e.g. TextOutput).  Device
 * memory for crp_run_device(), host memory for crp_run().  One record holds
 * the candidate index and its state at the moment of the action. */
typedef struct crp_records {
    uint64_t capacity;
    uint64_t *count;      /* records written (may exceed capacity: the rest were dropped) */
    uint64_t *index;      /* candidate index */
    int32_t *module;      /* module position in the chain */
    double *trajectory_length, *time;
    double *x, *y, *z;
    double *dx, *dy, *dz;
    double *energy;
    int32_t *id;
} crp_records;

enum crp_run_mode {
    CRP_MODE_AUTO = 0,
    CRP_MODE_CHUNKED = 1,   /* one thread per candidate, fixed steps per launch */
    CRP_MODE_PERSISTENT = 2 /* persistent CTAs refill lanes from a device queue */
};

typedef struct crp_run_opts {
    int32_t mode;
    int32_t block_size;        /* 0: autotuned; else a multiple of 32 up to 128 */
    int32_t ctas_per_sm;       /* 0: autotuned (persistent mode) */
    int32_t steps_per_launch;  /* 0: default (chunked mode) */
    int32_t refill_threshold;  /* persistent: lanes idle before a warp refills, 0: autotuned */
    int32_t budget_us;         /* persistent: device time per launch [us], 0: 200 ms */
    uint64_t max_steps;        /* per-candidate cap on accepted steps, 0: none */
    volatile int32_t *cancel;  /* host flag polled between launches, may be NULL */
    void *stream;              /* cudaStream_t, NULL: the legacy default stream */
    crp_records *records;      /* may be NULL */
} crp_run_opts;

typedef struct crp_run_stats {
    uint64_t particle_steps;    /* accepted propagation steps */
    uint64_t tries;             /* propagation tries including rejected ones */
    uint64_t field_evaluations; /* getField calls */
    uint64_t launches;          /* kernel launches of the stepping path (stepping kernels and
                                   the cell-ordering key kernels between them) */
    uint64_t active_left;       /* candidates still active on return */
    double device_ms;           /* device time of the stepping path: the stepping kernels and the
                                   cell ordering between them */
} crp_run_stats;

typedef struct crp_plan crp_plan;

/* Library and device */
uint32_t crp_abi_version(void);
crp_status crp_last_error(char *buffer, size_t size);
crp_status crp_device_count(int32_t *count);

/* Plan: validates the chain the way the reference constructors and setters
 * do (PropagationCK.cpp:163-190, PropagationBP.cpp:148-178,
 * DiffusionSDE.cpp:280-320), uploads grids and wave-mode tables to the
 * current device. */
crp_status crp_plan_create(const crp_plan_desc *desc, crp_plan **plan);
crp_status crp_plan_destroy(crp_plan *plan);

/* Run every active candidate until it is inactive (or max_steps).  Host
 * arrays: copied to the device and back inside the call; in the chunked mode,
 * from 2^18 candidates on, the inputs go in 8 chunks on a copy stream and the
 * first launch starts on each chunk as it arrives (the first launch's
 * device_ms then includes that wait).  Pinned host arrays give the fastest
 * copies. */
crp_status crp_run(crp_plan *plan, const crp_candidates *host, uint64_t n,
                   const crp_run_opts *opts, crp_run_stats *stats);
/* Same, on device-resident arrays, asynchronous with respect to the host
 * only where stats is NULL and no cancel flag is given. */
crp_status crp_run_device(crp_plan *plan, const crp_candidates *device, uint64_t n,
                          const crp_run_opts *opts, crp_run_stats *stats);

/* Launch-configuration autotuner.  Times short trials (at most
 * steps_per_candidate chain iterations each) on up to sample_n candidates
 * copied from the device arrays `device` (which stay unchanged): the chunked
 * launch, and persistent launches over CTAs per SM, refill threshold and
 * burst length.  The fastest is stored in the plan and used by runs whose
 * mode is CRP_MODE_AUTO; *result reports it.  No reference counterpart (the
 * reference's OpenMP schedule is fixed at build time, CMakeLists.txt:206). */
typedef struct crp_autotune_result {
    int32_t mode;              /* crp_run_mode chosen */
    int32_t ctas_per_sm;
    int32_t refill_threshold;
    int32_t burst;             /* chain iterations between refills */
    int32_t trials;
    int32_t _pad0;
    double steps_per_second;   /* of the chosen configuration on the sample */
    double chunked_steps_per_second;
} crp_autotune_result;

crp_status crp_autotune(crp_plan *plan, const crp_candidates *device, uint64_t n,
                        uint64_t sample_n, uint64_t steps_per_candidate, void *stream,
                        crp_autotune_result *result);

/* Field of the plan (sum of its components) at n positions (device arrays,
 * planar x[n] y[n] z[n] in and out).  MagneticField::getField. */
crp_status crp_field_eval(crp_plan *plan, uint64_t n, const double *pos_xyz,
                          double *b_xyz, void *stream);

/* ------------------------------------------------------------------------
 * Adjoint of the fixed-step Boris push (no reference counterpart)
 * ---------------------------------------------------------------------- */

/* Forward model: PropagationBP::dY (PropagationBP.cpp:19) with fixed step
 * `step` over one periodic Grid3f, the grid values taken as doubles with
 * double trilinear weights (the corner order of Grid.h:571), the direction
 * normalised after each step; n_steps steps.  Loss per candidate:
 * 1 - u_final . target.  The adjoint recomputes segments of
 * checkpoint_every (<= 128) steps from FP64 checkpoints. */
typedef struct crp_adjoint_desc {
    const float *grid_values; /* DEVICE pointer, Vector3f cells */
    uint64_t nx, ny, nz;
    double origin[3];
    double spacing[3];
    double step;              /* [m] */
    int32_t n_steps;
    int32_t checkpoint_every;
} crp_adjoint_desc;

/* Device arrays of n candidates (planar components). */
typedef struct crp_adjoint_io {
    uint64_t n;
    const double *x, *y, *z;       /* initial position [m] */
    const double *dx, *dy, *dz;    /* initial direction (unit) */
    const double *energy, *charge; /* [J], [C] */
    const double *tx, *ty, *tz;    /* target directions */
    double *loss;                  /* out: 1 - u_final . target */
    double *ux, *uy, *uz;          /* out: final direction (may be NULL) */
    double *grad_dx, *grad_dy, *grad_dz; /* out: dL/du0 */
    double *grad_energy;           /* out: dL/dE */
    double *grad_grid;             /* out: dL/d(grid value), nx*ny*nz*3, may be NULL */
} crp_adjoint_io;

/* Bytes of device workspace crp_bp_adjoint needs for n candidates. */
crp_status crp_bp_adjoint_workspace(const crp_adjoint_desc *desc, uint64_t n, size_t *bytes);
/* Forward pass only: loss (and final directions). */
crp_status crp_bp_forward_loss(const crp_adjoint_desc *desc, const crp_adjoint_io *io, void *stream);
/* Forward pass with checkpoints, then the reverse pass: loss and gradients.
 * The grid gradient is summed with 64-bit fixed-point atomics (unit
 * 2^-36 max|kappa|, kappa = q step c / 2E), so it is the same bits on every
 * run. */
crp_status crp_bp_adjoint(const crp_adjoint_desc *desc, const crp_adjoint_io *io, void *workspace,
                          size_t workspace_bytes, void *stream);
/* The two halves of crp_bp_adjoint: the forward pass that writes loss and
 * checkpoints into the workspace, and the reverse pass that reads them (same
 * desc, inputs and workspace, nothing changed in between). */
crp_status crp_bp_adjoint_forward(const crp_adjoint_desc *desc, const crp_adjoint_io *io,
                                  void *workspace, size_t workspace_bytes, void *stream);
crp_status crp_bp_adjoint_backward(const crp_adjoint_desc *desc, const crp_adjoint_io *io,
                                   void *workspace, size_t workspace_bytes, void *stream);

/* ------------------------------------------------------------------------
 * Allocation-free run
 * ---------------------------------------------------------------------- */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory -- a process whose device memory belongs to another allocator (a
 * framework's caching allocator that owns the device, a real-time loop that
 * must not block on the driver's allocator), a plugin limited to the buffers
 * its host hands it -- and so cannot create a crp_plan: a fixed-step
 * PropagationBP over one Grid3f whose values the caller already holds on the
 * device, followed by MaximumTrajectoryLength.  Nothing is allocated: the
 * run's scratch (counters and compaction lists) is a fixed static device
 * array that every device loading the library holds until exit, so one call
 * takes at most CRP_NOALLOC_MAX_CANDIDATES candidates (larger n returns
 * CRP_ERR_CAPACITY).  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), so make that first call before any stream
 * capture begins.  All calls share the array: calls whose work overlaps on
 * the GPU race on it.  Every candidate array, step_count (when given) and
 * grid_values must be device-reachable (CRP_ERR_INVALID_ARGUMENT otherwise);
 * spacing must be finite and > 0, step finite and > 0, max_length finite.
 * The call reads the run counters back to the host between launches and
 * returns when every candidate is inactive.  Results equal crp_run_device
 * with the same chain and precision. */
#define CRP_NOALLOC_MAX_CANDIDATES (1u << 20)

typedef struct crp_noalloc_grid_bp_desc {
    const float *grid_values; /* DEVICE pointer: nx*ny*nz cells of 3 floats, cell (ix, iy, iz) at
                                 index (ix*ny + iy)*nz + iz */
    uint64_t nx, ny, nz;
    double origin[3];
    double spacing[3];
    int32_t reflective;
    int32_t clip_volume;
    double step;             /* PropagationBP fixed step [m] */
    double max_length;       /* MaximumTrajectoryLength [m] */
    int32_t precision;       /* crp_precision */
    int32_t steps_per_launch; /* 0: default */
} crp_noalloc_grid_bp_desc;

crp_status crp_run_device_noalloc(const crp_noalloc_grid_bp_desc *desc,
                                  const crp_candidates *device, uint64_t n, void *stream,
                                  crp_run_stats *stats);

/* ------------------------------------------------------------------------
 * Host-side set-up and output (no device needed)
 * ---------------------------------------------------------------------- */

/* Charge of a particle id as ParticleState::setId assigns it
 * (ParticleState.cpp:50): Z*eplus for nuclei (negative for anti-nuclei),
 * HepPID charge for leptons, photons and neutrinos. */
crp_status crp_particle_charge(int32_t id, double *charge);

/* n draws of crpropa::Random seeded with seed (Random.cpp): kind 0 rand(),
 * 1 randUniform(a, b), 2 randVector() (3 values per draw), 3
 * randPowerLaw(a, b, c), 4 randNorm(), 6 randInt(). */
crp_status crp_random_draws(uint32_t seed, int32_t kind, uint64_t n, double a, double b,
                            double c, double *out);

/* The parameters JF12Field's constructor sets (variant 0, JF12Field.cpp:8),
 * PlanckJF12bField's (variant 1, JF12Field.cpp:352) or JF12FieldSolenoidal's
 * with its default arguments (variant 2), with the regular
 * field on and the striated and turbulent fields off, as constructed. */
crp_status crp_jf12_defaults(int32_t variant, crp_jf12_desc *out);

/* The parameters JF12FieldSolenoidal(delta, zs) sets (JF12FieldSolenoidal.cpp:8):
 * JF12Field's, with the disk's transition width delta and the X field's
 * scale height zs [m]; the arm crossings, the flux-closing eighth arm
 * strength and the azimuth integral's coefficients derived as the
 * constructor derives them.  Its setters change r1s / r2s (delta),
 * z_s (zs) and r2s = r2 (deactivateOuterTransition). */
crp_status crp_jf12_solenoidal(double delta, double zs, crp_jf12_desc *out);

/* The parameters UF23Field(model) sets (UF23Field.cpp:59-266). */
crp_status crp_uf23_defaults(int32_t model, crp_uf23_desc *out);

/* The state PT11Field() constructs (PT11Field.cpp:8: ASS disk and halo on). */
crp_status crp_pt11_defaults(crp_pt11_desc *out);

/* PT11Field::setUseASS / setUseBSS / setUseHalo (PT11Field.cpp:35-68):
 * switching the ASS or BSS disk on switches the other off and sets its pitch
 * and southern halo strength; switching a disk off changes nothing else. */
crp_status crp_pt11_use(crp_pt11_desc *io, int32_t which, int32_t use);

/* The state TF17Field(disk, halo) constructs (TF17Field.cpp:10-118: disk
 * and halo on). */
crp_status crp_tf17_defaults(int32_t disk, int32_t halo, crp_tf17_desc *out);

/* PolarizedSingleModeMagneticField(B_0, wavelength, sigma, r_0, e_1, e_2,
 * flagAmplitudeRms, flagPolarizationHelicity, flagMode)
 * (PolarizedSingleModeMagneticField.cpp:5-52): the constructor's checks
 * (CRP_ERR_INVALID_ARGUMENT with its message) and derived values. */
crp_status crp_single_mode_field(double b0, double wavelength, double sigma, const double r0[3],
                                 const double e1[3], const double e2[3], int32_t amplitude_rms,
                                 int32_t polarization_helicity, int32_t mode, crp_single_mode_desc *out);

/* The parameters KST24Field's constructor sets (KST24Field.cpp:15-124). */
crp_status crp_kst24_defaults(crp_kst24_desc *out);

/* CMZField() (CMZField.cpp:6, the intercloud field on, the others off) and the
 * objects of its four parts with the derived a, L and strengths as its
 * methods form them (CMZField.cpp:14-287). */
crp_status crp_cmz_defaults(crp_cmz_desc *out);

/* Turbulent Grid3f generation: GridTurbulence (GridTurbulence.cpp:29-123,
 * TurbulenceSpectrum), SimpleGridTurbulence (SimpleGridTurbulence.cpp:19-115,
 * power law k^alpha, alpha = -sindex - 2) and HelicalGridTurbulence
 * (HelicalGridTurbulence.cpp:19-127, helicity H). */
enum crp_turbulence_kind {
    CRP_TURBULENCE_GRID = 0,
    CRP_TURBULENCE_SIMPLE = 1,
    CRP_TURBULENCE_HELICAL = 2
};

typedef struct crp_turbulence_desc {
    int32_t kind;       /* crp_turbulence_kind */
    int32_t seed;       /* Random seed of the k-space draws; 0 is refused (the reference then seeds
                           from the system's entropy) */
    uint64_t n;         /* cells per side (GridProperties Nx = Ny = Nz) */
    double spacing;     /* cell size [m] */
    double brms, lmin, lmax; /* [T], [m], [m] */
    double lbendover, sindex, qindex; /* TurbulenceSpectrum (GridTurbulence); Simple and Helical
                                         use sindex only */
    double helicity;    /* HelicalGridTurbulence H, in [-1, 1] */
} crp_turbulence_desc;

/* The Random draws of the k-space loop for n_modes kept modes, in loop
 * order: GRID 2 per mode (rand theta, rand phase), SIMPLE 3 (rand theta,
 * randNorm amplitude, rand phase), HELICAL 3 (randNorm amplitude, rand
 * theta+, rand theta-). */
crp_status crp_turbulence_draws(uint32_t seed, int32_t kind, uint64_t n_modes, double *out);

/* Number of modes kept by the k-space loop (kMin <= |k| <= kMax). */
crp_status crp_turbulence_modes(const crp_turbulence_desc *d, uint64_t *n_modes);

/* A turbulent Grid3f generated on the device: the k-space amplitudes from
 * the reference's draws (host MT19937, crp_turbulence_draws), the inverse
 * real FFT (cuFFT, unnormalised as FFTW's) and the normalisation to brms
 * (scaleGrid(grid, Brms / rmsFieldStrength(grid)), GridTools.cpp:16, :59).
 * out: DEVICE memory for n^3 Vector3f cells (12 B each, Grid.h:338 order).
 * Allocates and frees its own scratch (k-space and FFT buffers).  FFTW is
 * not the FFT, so values equal the reference's in distribution, not bit for
 * bit. */
crp_status crp_turbulence_grid(const crp_turbulence_desc *d, float *out_device, void *stream);

/* Wave modes of PlaneWaveTurbulence(TurbulenceSpectrum(brms, lmin, lmax,
 * lbendover, sindex, qindex), nm, seed) (PlaneWaveTurbulence.cpp:79-229),
 * drawn with the reference's MT19937 sequence.  seed must be non-zero. */
crp_status crp_plane_wave_modes(double brms, double lmin, double lmax, double lbendover,
                                double sindex, double qindex, int32_t nm, int32_t seed,
                                double *xi, double *kappa, double *k, double *beta, double *ak);

/* A Source with SourceParticleType / SourceMultipleParticleTypes,
 * SourceEnergy or SourcePowerLawSpectrum, and SourceIsotropicEmission or
 * SourceDirection (Source.cpp:74-150, :742, :808), sampled in that feature
 * order from one crpropa::Random stream (Random::seedThreads(seed), one
 * thread). */
typedef struct crp_source_desc {
    int32_t n_types;
    int32_t spectrum;   /* 1: power law emin..emax with index; 0: fixed energy */
    const int32_t *ids;
    const double *abundances; /* NULL: equal */
    double emin, emax, index;
    double energy;
    int32_t isotropic;  /* 1: SourceIsotropicEmission; 0: direction[] */
    int32_t _pad0;
    double direction[3];
} crp_source_desc;

crp_status crp_source_sample(const crp_source_desc *src, uint32_t seed, uint64_t n, int32_t *id,
                             double *energy, double *dir_xyz /* planar x[n] y[n] z[n] */);

/* The same source features drawn on the device, for throughput runs that
 * should not copy candidates from the host (Source::getCandidate,
 * Source.cpp:22, with the features above).  Candidate first + i takes its
 * draws from a counter-based Philox4x32-10 stream keyed by seed, so a run
 * split over calls or ranks (first = the index of its first candidate) draws
 * the same candidates as one call; the distributions are the reference's,
 * the sequence is not MT19937's (crp_source_sample reproduces that).  id,
 * energy and dir_xyz (planar x[n] y[n] z[n]) are device arrays; stream is a
 * cudaStream_t (NULL: the legacy default stream); the call returns after the
 * launch.  1 to 256 particle types. */
crp_status crp_source_sample_device(const crp_source_desc *src, uint64_t seed, uint64_t first, uint64_t n,
                                    int32_t *id, double *energy, double *dir_xyz, void *stream);

/* Output columns (Output.h:76 OutputColumn, bit = enum value). */
enum crp_output_column {
    CRP_COL_TRAJECTORY_LENGTH = 0, CRP_COL_COLUMN_DENSITY = 1, CRP_COL_REDSHIFT = 2,
    CRP_COL_CURRENT_ID = 3, CRP_COL_CURRENT_ENERGY = 4, CRP_COL_CURRENT_POSITION = 5,
    CRP_COL_CURRENT_DIRECTION = 6, CRP_COL_SOURCE_ID = 7, CRP_COL_SOURCE_ENERGY = 8,
    CRP_COL_SOURCE_POSITION = 9, CRP_COL_SOURCE_DIRECTION = 10, CRP_COL_CREATED_ID = 11,
    CRP_COL_CREATED_ENERGY = 12, CRP_COL_CREATED_POSITION = 13, CRP_COL_CREATED_DIRECTION = 14,
    CRP_COL_CANDIDATE_TAG = 15, CRP_COL_SERIAL_NUMBER = 16, CRP_COL_WEIGHT = 17, CRP_COL_TIME = 18
};

typedef struct crp_output_desc {
    uint32_t columns;        /* bitset of crp_output_column */
    int32_t one_dimensional; /* Output::set1D */
    double length_scale, time_scale, energy_scale;
    const char *version;     /* "CRPropa version" header line */
} crp_output_desc;

/* Rows to print: one per detected candidate, vectors interleaved xyz. */
typedef struct crp_output_rows {
    const uint64_t *serial;
    const double *trajectory_length, *time;
    const int32_t *id;
    const double *energy, *position, *direction;
    const int32_t *source_id;
    const double *source_energy, *source_position, *source_direction;
    const double *weight; /* NULL: 1 */
} crp_output_rows;

/* TextOutput (TextOutput.cpp:55 printHeader, :166 process): write (or
 * append) n lines, optionally preceded by the header; a path ending in
 * ".gz" is written gzip-compressed (TextOutput.cpp:41, :388). */
crp_status crp_text_output_write(const char *path, int32_t append, int32_t header,
                                 const crp_output_desc *desc, uint64_t n,
                                 const crp_output_rows *rows);

#ifdef __cplusplus
}
#endif

#endif /* CRP_GPU_H */
