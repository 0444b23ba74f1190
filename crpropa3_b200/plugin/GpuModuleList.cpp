// GpuModuleList.cpp -- chain translation, candidate packing, device run
// through crp_gpu.h, write-back and host replay of the chain's actions.
#include "GpuModuleList.h"

#include "crp_gpu.h"

#include "crpropa/Geometry.h"
#include "crpropa/Grid.h"
#include "crpropa/Units.h"
#include "crpropa/magneticField/JF12Field.h"
#include "crpropa/magneticField/JF12FieldSolenoidal.h"
#include "crpropa/magneticField/MagneticFieldGrid.h"
#include "crpropa/magneticField/UF23Field.h"
#include "crpropa/magneticField/PT11Field.h"
#include "crpropa/magneticField/ArchimedeanSpiralField.h"
#include "crpropa/magneticField/TF17Field.h"
#include "crpropa/magneticField/PolarizedSingleModeMagneticField.h"
#include "crpropa/magneticField/KST24Field.h"
#include "crpropa/magneticField/CMZField.h"
#include "crpropa/magneticField/turbulentField/PlaneWaveTurbulence.h"
#include "crpropa/module/Boundary.h"
#include "crpropa/module/BreakCondition.h"
#include "crpropa/module/DiffusionSDE.h"
#include "crpropa/advectionField/AdvectionField.h"
#include "crpropa/advectionField/TimeDependentAdvectionField.h"
#include "crpropa/module/Observer.h"
#include "crpropa/module/Output.h"
#include "crpropa/module/PropagationBP.h"
#include "crpropa/module/PropagationCK.h"

#include <cxxabi.h>
#include <signal.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <typeinfo>
#include <vector>

using namespace crpropa;

namespace {

// ---------------------------------------------------------------------------
// Members the reference keeps private or protected without a getter.  An
// explicit instantiation may name any member regardless of access
// ([temp.explicit]); the friend function it defines hands out the member
// pointer.  Each use names the member exactly as the reference header
// declares it, so a change there fails this build instead of misreading.
template <typename Tag, typename Tag::type M>
struct Expose {
    friend typename Tag::type member(Tag) { return M; }
};

#define CRPGPU_MEMBER(TAG, CLASS, TYPE, NAME)      \
    struct TAG {                                    \
        typedef TYPE CLASS::*type;                  \
        friend type member(TAG);                    \
    };                                              \
    template struct Expose<TAG, &CLASS::NAME>

typedef std::vector<ref_ptr<ObserverFeature> > FeatureList;
typedef std::vector<ref_ptr<MagneticField> > FieldVector;

CRPGPU_MEMBER(ObserverFeatures, Observer, FeatureList, features);       // Observer.h:48
CRPGPU_MEMBER(ObserverAction, Observer, ref_ptr<Module>, detectionAction);
CRPGPU_MEMBER(ObserverClone, Observer, bool, clone);
CRPGPU_MEMBER(ObserverInactive, Observer, bool, makeInactive);
CRPGPU_MEMBER(ObserverFlagKey, Observer, std::string, flagKey);         // Observer.h:45
CRPGPU_MEMBER(ObserverFlagValue, Observer, std::string, flagValue);
CRPGPU_MEMBER(SurfaceOf, ObserverSurface, ref_ptr<Surface>, surface);  // Observer.h:92
CRPGPU_MEMBER(SphereCenter, Sphere, Vector3d, center);                 // Geometry.h:61
CRPGPU_MEMBER(SphereRadius, Sphere, double, radius);
CRPGPU_MEMBER(ListFields, MagneticFieldList, FieldVector, fields);     // MagneticField.h:82
CRPGPU_MEMBER(PeriodicInner, PeriodicMagneticField, ref_ptr<MagneticField>, field);  // :48
CRPGPU_MEMBER(WavesNm, PlaneWaveTurbulence, int, Nm);                  // PlaneWaveTurbulence.h:93
CRPGPU_MEMBER(WavesXi, PlaneWaveTurbulence, std::vector<Vector3d>, xi);
CRPGPU_MEMBER(WavesKappa, PlaneWaveTurbulence, std::vector<Vector3d>, kappa);
CRPGPU_MEMBER(WavesBeta, PlaneWaveTurbulence, std::vector<double>, beta);
CRPGPU_MEMBER(WavesAk, PlaneWaveTurbulence, std::vector<double>, Ak);
CRPGPU_MEMBER(WavesK, PlaneWaveTurbulence, std::vector<double>, k);
CRPGPU_MEMBER(RejectAction, AbstractCondition, ref_ptr<Module>, rejectAction);  // Module.h:39
CRPGPU_MEMBER(RejectInactive, AbstractCondition, bool, makeRejectedInactive);
CRPGPU_MEMBER(RejectKey, AbstractCondition, std::string, rejectFlagKey);
CRPGPU_MEMBER(RejectValue, AbstractCondition, std::string, rejectFlagValue);
CRPGPU_MEMBER(PlaneX0, Plane, Vector3d, x0);                           // Geometry.h:45
CRPGPU_MEMBER(PlaneN, Plane, Vector3d, n);
CRPGPU_MEMBER(BoxCorner, ParaxialBox, Vector3d, corner);               // Geometry.h:77
CRPGPU_MEMBER(BoxSize, ParaxialBox, Vector3d, size);
typedef double UF23Pars[26];
CRPGPU_MEMBER(ListInterruptAction, ModuleList, Output *, interruptAction);      // ModuleList.h:63
CRPGPU_MEMBER(ListHaveInterruptAction, ModuleList, bool, haveInterruptAction);
CRPGPU_MEMBER(UF23Model, UF23Field, const UF23Field::ModelType, fModelType);  // UF23Field.h
CRPGPU_MEMBER(UF23MaxR2, UF23Field, const double, fMaxRadiusSquared);
CRPGPU_MEMBER(UF23Parameters, UF23Field, UF23Pars, fParameters);
CRPGPU_MEMBER(UF23SinPitch, UF23Field, double, fSinPitch);
CRPGPU_MEMBER(UF23CosPitch, UF23Field, double, fCosPitch);
CRPGPU_MEMBER(UF23TanPitch, UF23Field, double, fTanPitch);
CRPGPU_MEMBER(PT11UseASS, PT11Field, bool, useASS);                    // PT11Field.h:28-46
CRPGPU_MEMBER(PT11UseBSS, PT11Field, bool, useBSS);
CRPGPU_MEMBER(PT11UseHalo, PT11Field, bool, useHalo);
#define CRPGPU_PT11(TAG, NAME) CRPGPU_MEMBER(TAG, PT11Field, double, NAME)
CRPGPU_PT11(PT11Pitch, pitch); CRPGPU_PT11(PT11CosPitch, cos_pitch); CRPGPU_PT11(PT11SinPitch, sin_pitch);
CRPGPU_PT11(PT11Phi, PHI); CRPGPU_PT11(PT11CosPhi, cos_PHI); CRPGPU_PT11(PT11D, d); CRPGPU_PT11(PT11RSun, R_sun);
CRPGPU_PT11(PT11Rc, R_c); CRPGPU_PT11(PT11Z0D, z0_D); CRPGPU_PT11(PT11B0D, B0_D); CRPGPU_PT11(PT11Z0H, z0_H);
CRPGPU_PT11(PT11R0H, R0_H); CRPGPU_PT11(PT11B0Hn, B0_Hn); CRPGPU_PT11(PT11B0Hs, B0_Hs);
CRPGPU_PT11(PT11Z11H, z11_H); CRPGPU_PT11(PT11Z12H, z12_H);
#undef CRPGPU_PT11
typedef std::vector<ref_ptr<AdvectionField> > AdvectionVector;
CRPGPU_MEMBER(AdvectionListFields, AdvectionFieldList, AdvectionVector, fields);  // AdvectionField.h:37
typedef double JF12Arms[11];
typedef double JF12Coeff[10];
CRPGPU_MEMBER(JF12CotPitch, JF12Field, double, cotPitch);                 // JF12Field.h:47-61
CRPGPU_MEMBER(JF12CotThetaX0, JF12Field, double, cotThetaX0);
CRPGPU_MEMBER(JF12BDisk, JF12Field, JF12Arms, bDisk);
CRPGPU_MEMBER(JF12SZs, JF12FieldSolenoidal, double, zS);                 // JF12FieldSolenoidal.h:35-55
CRPGPU_MEMBER(JF12SPhi0Arms, JF12FieldSolenoidal, JF12Arms, phi0Arms);
CRPGPU_MEMBER(JF12SPhiCoeff, JF12FieldSolenoidal, JF12Coeff, phiCoeff);
CRPGPU_MEMBER(JF12SR1, JF12FieldSolenoidal, double, r1);
CRPGPU_MEMBER(JF12SR2, JF12FieldSolenoidal, double, r2);
CRPGPU_MEMBER(JF12SR1s, JF12FieldSolenoidal, double, r1s);
CRPGPU_MEMBER(JF12SR2s, JF12FieldSolenoidal, double, r2s);
CRPGPU_MEMBER(TF17Disk, TF17Field, TF17DiskModel, disk_model);           // TF17Field.h:27-57
CRPGPU_MEMBER(TF17Halo, TF17Field, TF17HaloModel, halo_model);
CRPGPU_MEMBER(TF17UseDisk, TF17Field, bool, useDiskField);
CRPGPU_MEMBER(TF17UseHalo, TF17Field, bool, useHaloField);
#define CRPGPU_TF17(TAG, NAME) CRPGPU_MEMBER(TAG, TF17Field, double, NAME)
CRPGPU_TF17(TF17ADisk, a_disk); CRPGPU_TF17(TF17Z1Disk, z1_disk); CRPGPU_TF17(TF17R1Disk, r1_disk);
CRPGPU_TF17(TF17B1Disk, B1_disk); CRPGPU_TF17(TF17LDisk, L_disk); CRPGPU_TF17(TF17PhiDisk, phi_star_disk);
CRPGPU_TF17(TF17HDisk, H_disk); CRPGPU_TF17(TF17AHalo, a_halo); CRPGPU_TF17(TF17Z1Halo, z1_halo);
CRPGPU_TF17(TF17B1Halo, B1_halo); CRPGPU_TF17(TF17LHalo, L_halo); CRPGPU_TF17(TF17PhiHalo, phi_star_halo);
CRPGPU_TF17(TF17P0, p_0); CRPGPU_TF17(TF17CotP0, cot_p0); CRPGPU_TF17(TF17Hp, H_p); CRPGPU_TF17(TF17Lp, L_p);
CRPGPU_TF17(TF17Eps, epsilon);
#undef CRPGPU_TF17
// the derived state; the constructor stores no other argument (PolarizedSingleModeMagneticField.cpp:62-63)
CRPGPU_MEMBER(ModeU1, PolarizedSingleModeMagneticField, Vector3d, unitVector_1);  // PolarizedSingleModeMagneticField.h:34
CRPGPU_MEMBER(ModeU2, PolarizedSingleModeMagneticField, Vector3d, unitVector_2);
CRPGPU_MEMBER(ModeK, PolarizedSingleModeMagneticField, Vector3d, wavevector);
CRPGPU_MEMBER(ModeBMax, PolarizedSingleModeMagneticField, double, B_max);
CRPGPU_MEMBER(ModeSigma, PolarizedSingleModeMagneticField, double, sigma);
CRPGPU_MEMBER(ModeR0, PolarizedSingleModeMagneticField, Vector3d, r_0);
CRPGPU_MEMBER(TrackCenter, ObserverTracking, Vector3d, center);        // Observer.h:109
CRPGPU_MEMBER(TrackRadius, ObserverTracking, double, radius);
CRPGPU_MEMBER(TrackStep, ObserverTracking, double, stepSize);
CRPGPU_MEMBER(VetoId, ObserverParticleIdVeto, int, vetoParticleId);    // Observer.h:226
CRPGPU_MEMBER(CubeOrigin, CubicBoundary, Vector3d, origin);            // Boundary.h:104
CRPGPU_MEMBER(CubeSize, CubicBoundary, double, size);
CRPGPU_MEMBER(CubeMargin, CubicBoundary, double, margin);
CRPGPU_MEMBER(CubeLimit, CubicBoundary, bool, limitStep);
CRPGPU_MEMBER(SphCenter, SphericalBoundary, Vector3d, center);         // Boundary.h:136
CRPGPU_MEMBER(SphRadius, SphericalBoundary, double, radius);
CRPGPU_MEMBER(SphMargin, SphericalBoundary, double, margin);
CRPGPU_MEMBER(SphLimit, SphericalBoundary, bool, limitStep);
CRPGPU_MEMBER(EllF1, EllipsoidalBoundary, Vector3d, focalPoint1);      // Boundary.h:169
CRPGPU_MEMBER(EllF2, EllipsoidalBoundary, Vector3d, focalPoint2);
CRPGPU_MEMBER(EllAxis, EllipsoidalBoundary, double, majorAxis);
CRPGPU_MEMBER(EllMargin, EllipsoidalBoundary, double, margin);
CRPGPU_MEMBER(EllLimit, EllipsoidalBoundary, bool, limitStep);
CRPGPU_MEMBER(CylOrigin, CylindricalBoundary, Vector3d, origin);       // Boundary.h:204
CRPGPU_MEMBER(CylHeight, CylindricalBoundary, double, height);
CRPGPU_MEMBER(CylRadius, CylindricalBoundary, double, radius);
CRPGPU_MEMBER(CylMargin, CylindricalBoundary, double, margin);
CRPGPU_MEMBER(CylLimit, CylindricalBoundary, bool, limitStep);
// ParticleState::setDirection normalises (ParticleState.cpp:30); the device
// already wrote the normalised direction the reference would hold, and a
// second normalisation can move its last bit.
CRPGPU_MEMBER(StateDirection, ParticleState, Vector3d, direction);     // ParticleState.h:27

#undef CRPGPU_MEMBER

static_assert(sizeof(Vector3f) == 12, "Grid3f cells must be three packed floats (crp_grid3f_desc)");
static_assert(sizeof(float) == 4, "Grid1f cells must be single floats (crp_grid3f_desc)");

struct Unsupported : std::runtime_error {
    explicit Unsupported(const std::string &m) : std::runtime_error(m) {}
};

std::string type_name(const void *obj, const std::type_info &ti) {
    (void)obj;
    int st = 0;
    char *d = abi::__cxa_demangle(ti.name(), 0, 0, &st);
    std::string s = (st == 0 && d) ? d : ti.name();
    free(d);
    return s;
}

template <class T>
std::string name_of(const T *obj) {
    return type_name(obj, typeid(*obj));
}

// The advection field of a DiffusionSDE (exact types, AdvectionField.h:36-265)
// as crp_advection_desc entries of the module: a list becomes its fields in
// order (AdvectionFieldList::getField sums them, AdvectionField.cpp:12).
void addAdvection(const AdvectionField *f, crp_module_desc &d) {
    if (d.n_advection >= CRP_MAX_ADVECTION)
        throw Unsupported("DiffusionSDE with more than " + std::to_string(CRP_MAX_ADVECTION) + " advection fields");
    crp_advection_desc &A = d.advection[d.n_advection];
    std::memset(&A, 0, sizeof(A));
    auto origin = [&](const Vector3d &o) { A.origin[0] = o.x; A.origin[1] = o.y; A.origin[2] = o.z; };
    const std::type_info &t = typeid(*f);
    if (t == typeid(UniformAdvectionField)) {
        A.kind = CRP_ADVECTION_UNIFORM;  // a constant field: its value anywhere
        const Vector3d v = f->getField(Vector3d(0.), 0.);
        A.value[0] = v.x; A.value[1] = v.y; A.value[2] = v.z;
    } else if (t == typeid(ConstantSphericalAdvectionField)) {
        const ConstantSphericalAdvectionField *c = static_cast<const ConstantSphericalAdvectionField *>(f);
        A.kind = CRP_ADVECTION_CONSTANT_SPHERICAL;
        origin(c->getOrigin());
        A.v = c->getVWind();
    } else if (t == typeid(SphericalAdvectionField)) {
        const SphericalAdvectionField *c = static_cast<const SphericalAdvectionField *>(f);
        A.kind = CRP_ADVECTION_SPHERICAL;
        origin(c->getOrigin());
        A.radius = c->getRadius(); A.v = c->getVMax(); A.tau = c->getTau(); A.alpha = c->getAlpha();
    } else if (t == typeid(OneDimensionalCartesianShock)) {
        const OneDimensionalCartesianShock *c = static_cast<const OneDimensionalCartesianShock *>(f);
        A.kind = CRP_ADVECTION_CARTESIAN_SHOCK;
        A.compression = c->getComp(); A.v = c->getVup(); A.length = c->getShockwidth();
    } else if (t == typeid(OneDimensionalSphericalShock)) {
        const OneDimensionalSphericalShock *c = static_cast<const OneDimensionalSphericalShock *>(f);
        A.kind = CRP_ADVECTION_SPHERICAL_SHOCK_1D;
        A.radius = c->getShockRadius(); A.v = c->getVup(); A.compression = c->getComp();
        A.length = c->getShockwidth(); A.cool_upstream = c->getCooling() ? 1 : 0;
    } else if (t == typeid(ObliqueAdvectionShock)) {
        const ObliqueAdvectionShock *c = static_cast<const ObliqueAdvectionShock *>(f);
        A.kind = CRP_ADVECTION_OBLIQUE_SHOCK;
        A.compression = c->getComp(); A.v = c->getVup(); A.vy = c->getVy(); A.length = c->getShockwidth();
    } else if (t == typeid(SphericalAdvectionShock)) {
        const SphericalAdvectionShock *c = static_cast<const SphericalAdvectionShock *>(f);
        A.kind = CRP_ADVECTION_SPHERICAL_SHOCK;
        origin(c->getOrigin());
        A.radius = c->getR0(); A.v = c->getV0(); A.length = c->getLambda();
        A.r_rot = c->getRRot(); A.v_phi = c->getAzimuthalSpeed();
    } else if (t == typeid(OneDimensionalTimeDependentShock)) {
        const OneDimensionalTimeDependentShock *c = static_cast<const OneDimensionalTimeDependentShock *>(f);
        A.kind = CRP_ADVECTION_TIME_SHOCK;
        A.v = c->getVshock(); A.v1 = c->getV1(); A.v0 = c->getV0(); A.length = c->getShockWidth();
        A.t0 = c->getShockTime();
        A.x0 = c->getShockPosition(A.t0);  // x_sh0 + v_sh (t_sh0 - t_sh0)
    } else if (t == typeid(SedovTaylorBlastWave)) {
        const SedovTaylorBlastWave *c = static_cast<const SedovTaylorBlastWave *>(f);
        A.kind = CRP_ADVECTION_SEDOV_TAYLOR;
        A.energy = c->getEnergy(); A.density = c->getDensity(); A.length = c->getShockWidth();
    } else {
        throw Unsupported(name_of(f) + " (an advection field without a device form)");
    }
    d.n_advection++;
}

void translateAdvection(const AdvectionField *f, crp_module_desc &d) {
    if (typeid(*f) == typeid(AdvectionFieldList)) {
        const AdvectionFieldList *l = static_cast<const AdvectionFieldList *>(f);
        for (const ref_ptr<AdvectionField> &g : l->*member(AdvectionListFields())) {
            if (typeid(*g) == typeid(AdvectionFieldList)) throw Unsupported("a nested AdvectionFieldList");
            addAdvection(g.get(), d);
        }
    } else {
        addAdvection(f, d);
    }
}

std::string crp_error(crp_status st) {
    char buf[512];
    buf[0] = 0;
    crp_last_error(buf, sizeof(buf));
    std::ostringstream os;
    os << "GpuModuleList: device path failed (status " << int(st) << "): " << buf;
    return os.str();
}

void check(crp_status st) {
    if (st != CRP_OK) throw std::runtime_error(crp_error(st));
}

// One chain module's host-side actions, replayed from the device's records.
struct Action {
    int kind;  // CRP_MODULE_MAX_TRAJECTORY_LENGTH, CRP_MODULE_BOUNDARY or CRP_MODULE_OBSERVER
    const AbstractCondition *condition;
    const Observer *observer;
};

struct PeriodicWrap {
    Vector3d origin, extends;
    bool reflective;
};

// 64-bit FNV-1a over bytes, and a word-wise mix for large payloads.
struct Fingerprint {
    uint64_t h;
    Fingerprint() : h(1469598103934665603ull) {}
    void bytes(const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; i++) h = (h ^ c[i]) * 1099511628211ull;
    }
    template <class T>
    void value(const T &v) { bytes(&v, sizeof(v)); }
    void words(const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        size_t w = n / 8;
        uint64_t a = h;
        for (size_t i = 0; i < w; i++) {
            uint64_t x;
            std::memcpy(&x, c + 8 * i, 8);
            a = (a ^ x) * 0x9E3779B97F4A7C15ull;
            a ^= a >> 29;
        }
        h = a;
        bytes(c + 8 * w, n - 8 * w);
    }
};

struct Translation {
    std::vector<crp_field_component> fields;
    std::vector<crp_module_desc> modules;
    std::vector<Action> actions;  // one per modules[] entry
    std::deque<std::vector<double> > storage;  // push_back keeps references valid
    std::string perCandidateKey;
    bool hasPropagation;
    bool needsStepCount;
    Fingerprint fp;
    std::ostringstream text;

    Translation() : hasPropagation(false), needsStepCount(false) {}

    void addField(const MagneticField *f, const PeriodicWrap *wrap) {
        if (!f) throw Unsupported("a propagation module has no magnetic field");
        if (const MagneticFieldList *l = dynamic_cast<const MagneticFieldList *>(f)) {
            const FieldVector &v = l->*member(ListFields());
            for (size_t i = 0; i < v.size(); i++) addField(v[i].get(), wrap);
            return;
        }
        if (const PeriodicMagneticField *p = dynamic_cast<const PeriodicMagneticField *>(f)) {
            if (wrap) throw Unsupported("PeriodicMagneticField inside a PeriodicMagneticField");
            PeriodicMagneticField *q = const_cast<PeriodicMagneticField *>(p);
            PeriodicWrap w = {q->getOrigin(), q->getExtends(), q->isReflective()};
            addField((p->*member(PeriodicInner())).get(), &w);
            return;
        }
        crp_field_component c;
        std::memset(&c, 0, sizeof(c));
        if (wrap) {
            c.periodic = 1;
            c.periodic_reflective = wrap->reflective ? 1 : 0;
            for (int a = 0; a < 3; a++) {
                c.periodic_origin[a] = wrap->origin.data[a];
                c.periodic_extends[a] = wrap->extends.data[a];
            }
        }
        if (const MagneticFieldGrid *g = dynamic_cast<const MagneticFieldGrid *>(f)) {
            ref_ptr<Grid3f> grid = const_cast<MagneticFieldGrid *>(g)->getGrid();
            if (!grid.valid()) throw Unsupported("MagneticFieldGrid without a grid");
            c.kind = CRP_FIELD_GRID;
            text << "  field: ";
            fillGrid(*grid, 3, c.grid);
        } else if (const ModulatedMagneticFieldGrid *g =
                       dynamic_cast<const ModulatedMagneticFieldGrid *>(f)) {
            ModulatedMagneticFieldGrid *q = const_cast<ModulatedMagneticFieldGrid *>(g);
            ref_ptr<Grid3f> grid = q->getGrid();
            ref_ptr<Grid1f> mod = q->getModulationGrid();
            if (!grid.valid() || !mod.valid())
                throw Unsupported("ModulatedMagneticFieldGrid without a grid");
            c.kind = CRP_FIELD_MODULATED_GRID;
            text << "  field: ModulatedMagneticFieldGrid ";
            fillGrid(*grid, 3, c.grid);
            text << " modulation ";
            fillGrid(*mod, 1, c.modulation);
        } else if (typeid(*f) == typeid(JF12Field) || typeid(*f) == typeid(PlanckJF12bField) ||
                   typeid(*f) == typeid(JF12FieldSolenoidal)) {
            // exact types only: the parameters are the constructor's (JF12Field.cpp:8, :352),
            // which a subclass could change
            JF12Field *j = const_cast<JF12Field *>(static_cast<const JF12Field *>(f));
            const bool sol = typeid(*f) == typeid(JF12FieldSolenoidal);
            const int variant = typeid(*f) == typeid(PlanckJF12bField) ? CRP_JF12_PLANCK : CRP_JF12_JF12;
            if (crp_jf12_defaults(variant, &c.jf12) != CRP_OK) throw Unsupported("JF12Field parameters");
            if (sol) {  // JF12Field's constants and the solenoidal state as the object holds it
                const JF12FieldSolenoidal *s = static_cast<const JF12FieldSolenoidal *>(f);
                crp_jf12_desc &d = c.jf12;
                d.variant = CRP_JF12_SOLENOIDAL;
                d.cot_pitch = j->*member(JF12CotPitch());
                d.cot_theta_x0 = j->*member(JF12CotThetaX0());
                d.z_s = s->*member(JF12SZs());
                d.r1 = s->*member(JF12SR1());
                d.r2 = s->*member(JF12SR2());
                d.r1s = s->*member(JF12SR1s());
                d.r2s = s->*member(JF12SR2s());
                d.delta = d.r1s - d.r1;
                std::memcpy(d.phi0_arms, s->*member(JF12SPhi0Arms()), sizeof(d.phi0_arms));
                std::memcpy(d.b_arms, j->*member(JF12BDisk()), sizeof(d.b_arms));
                std::memcpy(d.phi_coeff, s->*member(JF12SPhiCoeff()), sizeof(d.phi_coeff));
            }
            c.kind = CRP_FIELD_JF12;
            c.jf12.use_regular = j->isUsingRegularField();
            c.jf12.use_disk = j->isUsingDiskField();
            c.jf12.use_toroidal_halo = j->isUsingToroidalHaloField();
            c.jf12.use_x = j->isUsingXField();
            c.jf12.use_striated = j->isUsingStriatedField();
            c.jf12.use_turbulent = j->isUsingTurbulentField();
            text << "  field: " << (sol ? "JF12FieldSolenoidal" : variant ? "PlanckJF12bField" : "JF12Field")
                 << " regular "
                 << c.jf12.use_regular << " disk " << c.jf12.use_disk << " halo " << c.jf12.use_toroidal_halo
                 << " X " << c.jf12.use_x;
            if (c.jf12.use_striated) {
                ref_ptr<Grid1f> g = j->getStriatedGrid();
                text << " striated ";
                fillGrid(*g, 1, c.modulation);
            }
            if (c.jf12.use_turbulent) {
                ref_ptr<Grid3f> g = j->getTurbulentGrid();
                text << " turbulent ";
                fillGrid(*g, 3, c.grid);
            }
        } else if (const UF23Field *u = dynamic_cast<const UF23Field *>(f)) {
            if (typeid(*f) != typeid(UF23Field)) throw Unsupported(name_of(f) + " (a UF23Field subclass)");
            crp_uf23_desc &d = c.uf23;
            c.kind = CRP_FIELD_UF23;
            d.model = (int32_t)(u->*member(UF23Model()));
            // the 26 parameters in UF23Field::EPar order, as crp_uf23_desc lays them out
            static_assert(offsetof(crp_uf23_desc, twisting_time) - offsetof(crp_uf23_desc, disk_b1) ==
                              25 * sizeof(double), "crp_uf23_desc parameter block");
            std::memcpy(&d.disk_b1, u->*member(UF23Parameters()), sizeof(UF23Pars));
            d.sin_pitch = u->*member(UF23SinPitch());
            d.cos_pitch = u->*member(UF23CosPitch());
            d.tan_pitch = u->*member(UF23TanPitch());
            d.max_radius_squared = u->*member(UF23MaxR2());
            d.kpc = kpc;
            d.microgauss = microgauss;
            text << "  field: UF23Field model " << d.model;
        } else if (const PT11Field *t = dynamic_cast<const PT11Field *>(f)) {
            if (typeid(*f) != typeid(PT11Field)) throw Unsupported(name_of(f) + " (a PT11Field subclass)");
            crp_pt11_desc &d = c.pt11;
            c.kind = CRP_FIELD_PT11;
            d.use_ass = t->*member(PT11UseASS()) ? 1 : 0;
            d.use_bss = t->*member(PT11UseBSS()) ? 1 : 0;
            d.use_halo = t->*member(PT11UseHalo()) ? 1 : 0;
            d.pitch = t->*member(PT11Pitch());
            d.cos_pitch = t->*member(PT11CosPitch());
            d.sin_pitch = t->*member(PT11SinPitch());
            d.phi = t->*member(PT11Phi());
            d.cos_phi = t->*member(PT11CosPhi());
            d.d = t->*member(PT11D());
            d.r_sun = t->*member(PT11RSun());
            d.r_c = t->*member(PT11Rc());
            d.z0_d = t->*member(PT11Z0D());
            d.b0_d = t->*member(PT11B0D());
            d.z0_h = t->*member(PT11Z0H());
            d.r0_h = t->*member(PT11R0H());
            d.b0_hn = t->*member(PT11B0Hn());
            d.b0_hs = t->*member(PT11B0Hs());
            d.z11_h = t->*member(PT11Z11H());
            d.z12_h = t->*member(PT11Z12H());
            text << "  field: PT11Field ass " << d.use_ass << " bss " << d.use_bss << " halo " << d.use_halo;
        } else if (const TF17Field *t = dynamic_cast<const TF17Field *>(f)) {
            if (typeid(*f) != typeid(TF17Field)) throw Unsupported(name_of(f) + " (a TF17Field subclass)");
            crp_tf17_desc &d = c.tf17;
            c.kind = CRP_FIELD_TF17;
            d.disk_model = (int32_t)(t->*member(TF17Disk()));
            d.halo_model = (int32_t)(t->*member(TF17Halo()));
            d.use_disk = t->*member(TF17UseDisk()) ? 1 : 0;
            d.use_halo = t->*member(TF17UseHalo()) ? 1 : 0;
            // every parameter as the object holds it (the ones its models do not
            // read may be uninitialised in the reference: the device does not read them either)
            d.a_disk = t->*member(TF17ADisk()); d.z1_disk = t->*member(TF17Z1Disk());
            d.r1_disk = t->*member(TF17R1Disk()); d.b1_disk = t->*member(TF17B1Disk());
            d.l_disk = t->*member(TF17LDisk()); d.phi_star_disk = t->*member(TF17PhiDisk());
            d.h_disk = t->*member(TF17HDisk()); d.a_halo = t->*member(TF17AHalo());
            d.z1_halo = t->*member(TF17Z1Halo()); d.b1_halo = t->*member(TF17B1Halo());
            d.l_halo = t->*member(TF17LHalo()); d.phi_star_halo = t->*member(TF17PhiHalo());
            d.p0 = t->*member(TF17P0()); d.cot_p0 = t->*member(TF17CotP0());
            d.h_p = t->*member(TF17Hp()); d.l_p = t->*member(TF17Lp());
            d.epsilon = t->*member(TF17Eps());
            text << "  field: TF17Field disk " << t->getDiskModel() << " halo " << t->getHaloModel()
                 << " use disk " << d.use_disk << " halo " << d.use_halo;
        } else if (const PolarizedSingleModeMagneticField *s =
                       dynamic_cast<const PolarizedSingleModeMagneticField *>(f)) {
            if (typeid(*f) != typeid(PolarizedSingleModeMagneticField))
                throw Unsupported(name_of(f) + " (a PolarizedSingleModeMagneticField subclass)");
            crp_single_mode_desc &d = c.single_mode;
            c.kind = CRP_FIELD_SINGLE_MODE;
            const Vector3d &u1 = s->*member(ModeU1()), &u2 = s->*member(ModeU2()), &k = s->*member(ModeK()),
                           &r0 = s->*member(ModeR0());
            const double v[4][3] = {{u1.x, u1.y, u1.z}, {u2.x, u2.y, u2.z}, {k.x, k.y, k.z}, {r0.x, r0.y, r0.z}};
            for (int a = 0; a < 3; a++) { d.u1[a] = v[0][a]; d.u2[a] = v[1][a]; d.k[a] = v[2][a]; d.r0[a] = v[3][a]; }
            d.b_max = s->*member(ModeBMax());
            d.sigma = s->*member(ModeSigma());
            text << "  field: PolarizedSingleModeMagneticField sigma " << d.sigma;
        } else if (typeid(*f) == typeid(KST24Field)) {
            // exact type: no setters, every parameter is the constructor's (KST24Field.cpp:15-124)
            if (crp_kst24_defaults(&c.kst24) != CRP_OK) throw Unsupported("KST24Field parameters");
            c.kind = CRP_FIELD_KST24;
            text << "  field: KST24Field";
        } else if (typeid(*f) == typeid(CMZField)) {
            // exact type: the objects are the methods' constants (CMZField.cpp:116-287), the switches the object's
            const CMZField *z = static_cast<const CMZField *>(f);
            if (crp_cmz_defaults(&c.cmz) != CRP_OK) throw Unsupported("CMZField parameters");
            c.kind = CRP_FIELD_CMZ;
            c.cmz.use_mc = z->getUseMCField();
            c.cmz.use_ic = z->getUseICField();
            c.cmz.use_ntf = z->getUseNTFField();
            c.cmz.use_radio_arc = z->getUseRadioArc();
            text << "  field: CMZField MC " << c.cmz.use_mc << " IC " << c.cmz.use_ic << " NTF " << c.cmz.use_ntf
                 << " radio arc " << c.cmz.use_radio_arc;
        } else if (const ArchimedeanSpiralField *a = dynamic_cast<const ArchimedeanSpiralField *>(f)) {
            if (typeid(*f) != typeid(ArchimedeanSpiralField))
                throw Unsupported(name_of(f) + " (an ArchimedeanSpiralField subclass)");
            c.kind = CRP_FIELD_ARCHIMEDEAN_SPIRAL;
            c.archimedean.b0 = a->getB0();
            c.archimedean.r0 = a->getR0();
            c.archimedean.omega = a->getOmega();
            c.archimedean.vw = a->getVw();
            text << "  field: ArchimedeanSpiralField";
        } else if (const PlaneWaveTurbulence *w = dynamic_cast<const PlaneWaveTurbulence *>(f)) {
            const int nm = w->*member(WavesNm());
            const std::vector<Vector3d> &xi = w->*member(WavesXi());
            const std::vector<Vector3d> &kap = w->*member(WavesKappa());
            storage.push_back(std::vector<double>(3 * nm));
            std::vector<double> &xs = storage.back();
            storage.push_back(std::vector<double>(3 * nm));
            std::vector<double> &ks = storage.back();
            for (int i = 0; i < nm; i++)
                for (int a = 0; a < 3; a++) {
                    xs[3 * i + a] = xi[i].data[a];
                    ks[3 * i + a] = kap[i].data[a];
                }
            storage.push_back(w->*member(WavesK()));
            const std::vector<double> &kk = storage.back();
            storage.push_back(w->*member(WavesBeta()));
            const std::vector<double> &bb = storage.back();
            storage.push_back(w->*member(WavesAk()));
            const std::vector<double> &aa = storage.back();
            c.kind = CRP_FIELD_PLANE_WAVE;
            c.plane_wave.n_modes = nm;
            c.plane_wave.xi = &xs[0];
            c.plane_wave.kappa = &ks[0];
            c.plane_wave.k = &kk[0];
            c.plane_wave.beta = &bb[0];
            c.plane_wave.ak = &aa[0];
            fp.words(&xs[0], 8 * xs.size());
            fp.words(&ks[0], 8 * ks.size());
            fp.words(&kk[0], 8 * kk.size());
            fp.words(&bb[0], 8 * bb.size());
            fp.words(&aa[0], 8 * aa.size());
            text << "  field: PlaneWaveTurbulence " << nm << " modes";
        } else if (const UniformMagneticField *u = dynamic_cast<const UniformMagneticField *>(f)) {
            Vector3d b = u->getField(Vector3d(0.));
            c.kind = CRP_FIELD_UNIFORM;
            for (int a = 0; a < 3; a++) c.uniform[a] = b.data[a];
            text << "  field: UniformMagneticField " << b.x << " " << b.y << " " << b.z;
        } else if (const crpgpu::ToroidalMagneticField *t =
                       dynamic_cast<const crpgpu::ToroidalMagneticField *>(f)) {
            c.kind = CRP_FIELD_TOROIDAL;
            c.toroidal_b0 = t->getB0();
            text << "  field: ToroidalMagneticField b0 " << c.toroidal_b0;
        } else {
            throw Unsupported("magnetic field " + name_of(f) + " has no device form");
        }
        if (wrap)
            text << " in PeriodicMagneticField extends " << wrap->extends.x << " reflective "
                 << wrap->reflective;
        text << "\n";
        fields.push_back(c);
    }

    // A Grid3f (width 3) or Grid1f (width 1) as a crp_grid3f_desc over the
    // grid's own storage (Grid.h:161-336: origin, spacing, boundary flags,
    // interpolation type).
    template <typename T>
    void fillGrid(Grid<T> &grid, int width, crp_grid3f_desc &d) {
        std::vector<T> &v = grid.getGrid();
        if (v.empty()) throw Unsupported("empty grid");
        const interpolationType ip = grid.getInterpolationType();
        if (ip != TRILINEAR && ip != TRICUBIC && ip != NEAREST_NEIGHBOUR)
            throw Unsupported("grid interpolation " + grid.getInterpolationTypeName());
        d.values = reinterpret_cast<const float *>(&v[0]);
        d.nx = grid.getNx();
        d.ny = grid.getNy();
        d.nz = grid.getNz();
        Vector3d o = grid.getOrigin(), s = grid.getSpacing();
        for (int a = 0; a < 3; a++) {
            d.origin[a] = o.data[a];
            d.spacing[a] = s.data[a];
        }
        d.reflective = grid.isReflective() ? 1 : 0;
        d.clip_volume = grid.getClipVolume() ? 1 : 0;
        d.interpolation = (int32_t)ip;
        fp.words(d.values, sizeof(float) * width * v.size());
        text << (width == 3 ? "Grid3f " : "Grid1f ") << d.nx << "x" << d.ny << "x" << d.nz << " spacing "
             << s.x << " reflective " << d.reflective << " clipVolume " << d.clip_volume << " "
             << grid.getInterpolationTypeName();
    }

    void setField(const MagneticField *f) {
        if (hasPropagation) throw Unsupported("more than one propagation module");
        hasPropagation = true;
        addField(f, 0);
    }

    static crp_module_desc blank(int kind) {
        crp_module_desc m;
        std::memset(&m, 0, sizeof(m));
        m.kind = kind;
        m.deactivate_on_detection = 1;
        return m;
    }

    void addModule(const Module *m) {
        if (const PropagationBP *p = dynamic_cast<const PropagationBP *>(m)) {
            crp_module_desc d = blank(CRP_MODULE_PROPAGATION);
            d.propagator = CRP_PROP_BP;
            d.tolerance = p->getTolerance();
            d.min_step = p->getMinimumStep();
            d.max_step = p->getMaximumStep();
            text << "  module: PropagationBP tolerance " << d.tolerance << " minStep " << d.min_step
                 << " maxStep " << d.max_step << "\n";
            setField(p->getField().get());
            push(d, Action());
        } else if (const PropagationCK *p = dynamic_cast<const PropagationCK *>(m)) {
            crp_module_desc d = blank(CRP_MODULE_PROPAGATION);
            d.propagator = CRP_PROP_CK;
            d.tolerance = p->getTolerance();
            d.min_step = p->getMinimumStep();
            d.max_step = p->getMaximumStep();
            text << "  module: PropagationCK tolerance " << d.tolerance << " minStep " << d.min_step
                 << " maxStep " << d.max_step << "\n";
            setField(p->getField().get());
            push(d, Action());
        } else if (const DiffusionSDE *p = dynamic_cast<const DiffusionSDE *>(m)) {
            crp_module_desc d = blank(CRP_MODULE_PROPAGATION);
            if (p->getAdvectionField().valid()) translateAdvection(p->getAdvectionField().get(), d);
            d.propagator = CRP_PROP_SDE;
            d.tolerance = p->getTolerance();
            d.min_step = p->getMinimumStep();
            d.max_step = p->getMaximumStep();
            d.sde_epsilon = p->getEpsilon();
            d.sde_alpha = p->getAlpha();
            d.sde_scale = p->getScale();
            text << "  module: DiffusionSDE tolerance " << d.tolerance << " minStep " << d.min_step
                 << " maxStep " << d.max_step << " epsilon " << d.sde_epsilon << " alpha "
                 << d.sde_alpha << " scale " << d.sde_scale << "\n";
            setField(p->getMagneticField().get());
            needsStepCount = true;
            push(d, Action());
        } else if (const crpgpu::CandidateMaximumTrajectoryLength *c =
                       dynamic_cast<const crpgpu::CandidateMaximumTrajectoryLength *>(m)) {
            if (!perCandidateKey.empty() && perCandidateKey != c->getPropertyKey())
                throw Unsupported("two CandidateMaximumTrajectoryLength modules with different keys");
            perCandidateKey = c->getPropertyKey();
            crp_module_desc d = blank(CRP_MODULE_MAX_TRAJECTORY_LENGTH);
            d.per_candidate_length = 1;
            d.record = 1;
            condition(c);
            text << "  module: CandidateMaximumTrajectoryLength key " << perCandidateKey << "\n";
            Action a = {CRP_MODULE_MAX_TRAJECTORY_LENGTH, c, 0};
            push(d, a);
        } else if (const MaximumTrajectoryLength *c = dynamic_cast<const MaximumTrajectoryLength *>(m)) {
            if (!c->getObserverPositions().empty())
                throw Unsupported("MaximumTrajectoryLength with observer positions");
            crp_module_desc d = blank(CRP_MODULE_MAX_TRAJECTORY_LENGTH);
            d.max_length = c->getMaximumTrajectoryLength();
            d.record = 1;
            condition(c);
            text << "  module: MaximumTrajectoryLength " << d.max_length << "\n";
            Action a = {CRP_MODULE_MAX_TRAJECTORY_LENGTH, c, 0};
            push(d, a);
        } else if (const Observer *o = dynamic_cast<const Observer *>(m)) {
            const FeatureList &fs = o->*member(ObserverFeatures());
            if (fs.empty()) {
                text << "  module: Observer without features (never detects; dropped)\n";
                return;
            }
            if (fs.size() > CRP_MAX_OBSERVER_FEATURES)
                throw Unsupported("Observer with more than 4 features");
            crp_module_desc d = blank(CRP_MODULE_OBSERVER);
            d.n_features = int32_t(fs.size());
            text << "  module: Observer";
            for (size_t k = 0; k < fs.size(); k++) {
                feature(fs[k].get(), d.features[k]);
                text << (k ? ", " : " ");
            }
            d.deactivate_on_detection = (o->*member(ObserverInactive())) ? 1 : 0;
            d.record = 1;
            const Module *act = (o->*member(ObserverAction())).get();
            text << " deactivate " << d.deactivate_on_detection << " action "
                 << (act ? name_of(act) : std::string("none")) << "\n";
            Action ac = {CRP_MODULE_OBSERVER, 0, o};
            push(d, ac);
        } else if (dynamic_cast<const CubicBoundary *>(m) || dynamic_cast<const SphericalBoundary *>(m) ||
                   dynamic_cast<const EllipsoidalBoundary *>(m) || dynamic_cast<const CylindricalBoundary *>(m)) {
            const AbstractCondition *c = dynamic_cast<const AbstractCondition *>(m);
            crp_module_desc d = blank(CRP_MODULE_BOUNDARY);
            d.record = 1;
            condition(c);
            Vector3d a0, b0;
            if (const CubicBoundary *q = dynamic_cast<const CubicBoundary *>(m)) {
                d.boundary = CRP_BOUNDARY_CUBIC;
                a0 = q->*member(CubeOrigin());
                d.boundary_size = q->*member(CubeSize());
                d.boundary_margin = q->*member(CubeMargin());
                d.boundary_limit_step = (q->*member(CubeLimit())) ? 1 : 0;
                text << "  module: CubicBoundary size " << d.boundary_size;
            } else if (const SphericalBoundary *q = dynamic_cast<const SphericalBoundary *>(m)) {
                d.boundary = CRP_BOUNDARY_SPHERICAL;
                a0 = q->*member(SphCenter());
                d.boundary_size = q->*member(SphRadius());
                d.boundary_margin = q->*member(SphMargin());
                d.boundary_limit_step = (q->*member(SphLimit())) ? 1 : 0;
                text << "  module: SphericalBoundary radius " << d.boundary_size;
            } else if (const EllipsoidalBoundary *q = dynamic_cast<const EllipsoidalBoundary *>(m)) {
                d.boundary = CRP_BOUNDARY_ELLIPSOIDAL;
                a0 = q->*member(EllF1());
                b0 = q->*member(EllF2());
                d.boundary_size = q->*member(EllAxis());
                d.boundary_margin = q->*member(EllMargin());
                d.boundary_limit_step = (q->*member(EllLimit())) ? 1 : 0;
                text << "  module: EllipsoidalBoundary major axis " << d.boundary_size;
            } else {
                const CylindricalBoundary *cy = dynamic_cast<const CylindricalBoundary *>(m);
                d.boundary = CRP_BOUNDARY_CYLINDRICAL;
                a0 = cy->*member(CylOrigin());
                d.boundary_size = cy->*member(CylHeight());
                d.boundary_radius = cy->*member(CylRadius());
                d.boundary_margin = cy->*member(CylMargin());
                d.boundary_limit_step = (cy->*member(CylLimit())) ? 1 : 0;
                text << "  module: CylindricalBoundary height " << d.boundary_size << " radius "
                     << d.boundary_radius;
            }
            for (int k = 0; k < 3; k++) {
                d.boundary_a[k] = a0.data[k];
                d.boundary_b[k] = b0.data[k];
            }
            text << " margin " << d.boundary_margin << " limitStep " << d.boundary_limit_step << "\n";
            Action ac = {CRP_MODULE_BOUNDARY, c, 0};
            push(d, ac);
        } else {
            throw Unsupported("module " + name_of(m) + " has no device form");
        }
    }

    // One ObserverFeature; exact classes only (a subclass may override checkDetection).
    void feature(const ObserverFeature *f, crp_observer_feature_desc &fd) {
        std::memset(&fd, 0, sizeof(fd));
        const std::type_info &ti = typeid(*f);
        if (const ObserverSurface *sf = dynamic_cast<const ObserverSurface *>(f)) {
            if (ti != typeid(ObserverSurface)) throw Unsupported("observer feature " + name_of(f) + " has no device form");
            const Surface *surf = (sf->*member(SurfaceOf())).get();
            Vector3d a, b;
            double r = 0;
            if (surf && typeid(*surf) == typeid(Sphere)) {
                const Sphere *sp = static_cast<const Sphere *>(surf);
                fd.kind = CRP_OBSERVER_SURFACE_SPHERE;
                a = sp->*member(SphereCenter());
                r = sp->*member(SphereRadius());
                text << "ObserverSurface(Sphere center " << a.x << " " << a.y << " " << a.z << " radius " << r << ")";
            } else if (surf && typeid(*surf) == typeid(Plane)) {
                const Plane *pl = static_cast<const Plane *>(surf);
                fd.kind = CRP_OBSERVER_SURFACE_PLANE;
                a = pl->*member(PlaneX0());
                b = pl->*member(PlaneN());
                text << "ObserverSurface(Plane)";
            } else if (surf && typeid(*surf) == typeid(ParaxialBox)) {
                const ParaxialBox *bx = static_cast<const ParaxialBox *>(surf);
                fd.kind = CRP_OBSERVER_SURFACE_BOX;
                a = bx->*member(BoxCorner());
                b = bx->*member(BoxSize());
                text << "ObserverSurface(ParaxialBox)";
            } else {
                throw Unsupported("ObserverSurface over " + (surf ? name_of(surf) : std::string("nothing")));
            }
            for (int k = 0; k < 3; k++) {
                fd.a[k] = a.data[k];
                fd.b[k] = b.data[k];
            }
            fd.r = r;
        } else if (ti == typeid(ObserverDetectAll)) {
            fd.kind = CRP_OBSERVER_DETECT_ALL;
            text << "ObserverDetectAll";
        } else if (ti == typeid(ObserverTracking)) {
            const ObserverTracking *t = static_cast<const ObserverTracking *>(f);
            fd.kind = CRP_OBSERVER_TRACKING;
            const Vector3d &c = t->*member(TrackCenter());
            for (int k = 0; k < 3; k++) fd.a[k] = c.data[k];
            fd.r = t->*member(TrackRadius());
            fd.step = t->*member(TrackStep());
            text << "ObserverTracking";
        } else if (ti == typeid(Observer1D)) {
            fd.kind = CRP_OBSERVER_1D;
            text << "Observer1D";
        } else if (ti == typeid(ObserverInactiveVeto)) {
            fd.kind = CRP_OBSERVER_INACTIVE_VETO;
            text << "ObserverInactiveVeto";
        } else if (ti == typeid(ObserverNucleusVeto)) {
            fd.kind = CRP_OBSERVER_NUCLEUS_VETO;
            text << "ObserverNucleusVeto";
        } else if (ti == typeid(ObserverNeutrinoVeto)) {
            fd.kind = CRP_OBSERVER_NEUTRINO_VETO;
            text << "ObserverNeutrinoVeto";
        } else if (ti == typeid(ObserverPhotonVeto)) {
            fd.kind = CRP_OBSERVER_PHOTON_VETO;
            text << "ObserverPhotonVeto";
        } else if (ti == typeid(ObserverElectronVeto)) {
            fd.kind = CRP_OBSERVER_ELECTRON_VETO;
            text << "ObserverElectronVeto";
        } else if (ti == typeid(ObserverParticleIdVeto)) {
            fd.kind = CRP_OBSERVER_PARTICLE_ID_VETO;
            fd.particle_id = static_cast<const ObserverParticleIdVeto *>(f)->*member(VetoId());
            text << "ObserverParticleIdVeto " << fd.particle_id;
        } else {
            throw Unsupported("observer feature " + name_of(f) + " has no device form");
        }
    }

    void condition(const AbstractCondition *c) {
        if (!(c->*member(RejectInactive())))
            throw Unsupported(name_of(c) + " with setMakeRejectedInactive(false)");
    }

    void push(const crp_module_desc &d, const Action &a) {
        modules.push_back(d);
        actions.push_back(a);
        fp.value(d);
    }

    void finish(int precision, uint64_t seed) {
        if (!hasPropagation) throw Unsupported("no propagation module");
        fp.value(precision);
        fp.value(seed);
        for (size_t i = 0; i < fields.size(); i++) {
            crp_field_component c = fields[i];
            c.grid.values = c.modulation.values = 0;  // content hashed above
            c.plane_wave.xi = c.plane_wave.kappa = c.plane_wave.k = c.plane_wave.beta =
                c.plane_wave.ak = 0;
            fp.value(c);
        }
    }
};

volatile int32_t g_cancel = 0;

extern "C" void crpgpu_on_signal(int sig) { g_cancel = sig; }

struct SignalScope {
    struct sigaction old_int, old_term;
    SignalScope() {
        g_cancel = 0;
        struct sigaction sa;
        std::memset(&sa, 0, sizeof(sa));
        sa.sa_handler = crpgpu_on_signal;
        sigaction(SIGINT, &sa, &old_int);
        sigaction(SIGTERM, &sa, &old_term);
    }
    ~SignalScope() {
        sigaction(SIGINT, &old_int, 0);
        sigaction(SIGTERM, &old_term, 0);
    }
};

// Host structure-of-arrays of one batch.
struct Batch {
    std::vector<int32_t> id;
    std::vector<double> charge, energy, x, y, z, dx, dy, dz, px, py, pz, length, time, cur, next,
        max_length;
    std::vector<uint8_t> active;
    std::vector<uint32_t> flags;
    std::vector<uint64_t> steps;

    void resize(size_t n, bool per, bool sc) {
        id.resize(n);
        std::vector<double> *d[] = {&charge, &energy, &x, &y, &z, &dx, &dy, &dz, &px, &py, &pz,
                                    &length, &time, &cur, &next};
        for (size_t i = 0; i < sizeof(d) / sizeof(d[0]); i++) d[i]->resize(n);
        max_length.resize(per ? n : 0);
        active.resize(n);
        flags.resize(n);
        steps.resize(sc ? n : 0);
    }

    crp_candidates view() {
        crp_candidates c;
        std::memset(&c, 0, sizeof(c));
        c.id = &id[0];
        c.charge = &charge[0];
        c.energy = &energy[0];
        c.x = &x[0]; c.y = &y[0]; c.z = &z[0];
        c.dx = &dx[0]; c.dy = &dy[0]; c.dz = &dz[0];
        c.px = &px[0]; c.py = &py[0]; c.pz = &pz[0];
        c.trajectory_length = &length[0];
        c.time = &time[0];
        c.current_step = &cur[0];
        c.next_step = &next[0];
        c.active = &active[0];
        c.flags = &flags[0];
        c.max_length = max_length.empty() ? 0 : &max_length[0];
        c.step_count = steps.empty() ? 0 : &steps[0];
        return c;
    }
};

struct Records {
    uint64_t count;
    std::vector<uint64_t> index;
    std::vector<int32_t> module, id;
    std::vector<double> length, time, x, y, z, dx, dy, dz, energy;

    crp_records view(uint64_t cap) {
        index.resize(cap); module.resize(cap); id.resize(cap);
        std::vector<double> *d[] = {&length, &time, &x, &y, &z, &dx, &dy, &dz, &energy};
        for (size_t i = 0; i < sizeof(d) / sizeof(d[0]); i++) d[i]->resize(cap);
        crp_records r;
        std::memset(&r, 0, sizeof(r));
        count = 0;
        r.capacity = cap;
        r.count = &count;
        r.index = &index[0]; r.module = &module[0]; r.id = &id[0];
        r.trajectory_length = &length[0]; r.time = &time[0];
        r.x = &x[0]; r.y = &y[0]; r.z = &z[0];
        r.dx = &dx[0]; r.dy = &dy[0]; r.dz = &dz[0];
        r.energy = &energy[0];
        return r;
    }
};

void set_direction_exact(ParticleState &s, double x, double y, double z) {
    s.*member(StateDirection()) = Vector3d(x, y, z);
}

}  // namespace

namespace crpgpu {

// ---------------------------------------------------------------------------
ToroidalMagneticField::ToroidalMagneticField(double b0) : b0(b0) {}

Vector3d ToroidalMagneticField::getField(const Vector3d &p) const {
    double r = std::sqrt(p.x * p.x + p.y * p.y);
    return Vector3d(-p.y, p.x, 0.) * (b0 / r);
}

double ToroidalMagneticField::getB0() const { return b0; }

CandidateMaximumTrajectoryLength::CandidateMaximumTrajectoryLength(const std::string &key)
    : key(key) {}

void CandidateMaximumTrajectoryLength::process(Candidate *c) const {
    double maxLength = c->getProperty(key).asDouble();
    double length = c->getTrajectoryLength();
    if (length >= maxLength)
        reject(c);
    else
        c->limitNextStep(maxLength - length);
}

std::string CandidateMaximumTrajectoryLength::getPropertyKey() const { return key; }

std::string CandidateMaximumTrajectoryLength::getDescription() const {
    return "Maximum trajectory length from candidate property " + key;
}

// ---------------------------------------------------------------------------
struct GpuModuleList::Impl {
    int precision;
    uint64_t seed;
    size_t batch;
    bool cpuFallback;
    crp_plan *plan;
    uint64_t planFingerprint;
    crp_run_stats stats;
    uint64_t events;
    double eventsPerCandidate;  // most records per candidate seen by this plan's runs

    Impl() : precision(CRP_PRECISION_FP64), seed(0), batch(size_t(1) << 20), cpuFallback(false),
             plan(0), planFingerprint(0), events(0), eventsPerCandidate(0) {
        std::memset(&stats, 0, sizeof(stats));
    }
    ~Impl() {
        if (plan) crp_plan_destroy(plan);
    }
};

GpuModuleList::GpuModuleList() : impl(new Impl()) {}

GpuModuleList::~GpuModuleList() { delete impl; }

void GpuModuleList::setPrecision(Precision p) { impl->precision = p; }

GpuModuleList::Precision GpuModuleList::getPrecision() const {
    return impl->precision == CRP_PRECISION_MIXED ? MIXED : FP64;
}

void GpuModuleList::setSeed(uint64_t seed) { impl->seed = seed; }

void GpuModuleList::setBatchSize(size_t n) {
    if (n == 0) throw std::runtime_error("GpuModuleList: batch size must be positive");
    impl->batch = n;
}

void GpuModuleList::setCpuFallback(bool allow) { impl->cpuFallback = allow; }

const crp_run_stats &GpuModuleList::getLastRunStats() const { return impl->stats; }

uint64_t GpuModuleList::getLastRunEvents() const { return impl->events; }

static void translate(const ModuleList &ml, int precision, uint64_t seed, Translation &t) {
    for (ModuleList::const_iterator it = ml.begin(); it != ml.end(); ++it) t.addModule(it->get());
    t.finish(precision, seed);
}

bool GpuModuleList::isSupported(std::string *reason) const {
    try {
        Translation t;
        translate(*this, impl->precision, impl->seed, t);
        return true;
    } catch (Unsupported &e) {
        if (reason) *reason = e.what();
        return false;
    }
}

std::string GpuModuleList::describePlan() const {
    Translation t;
    try {
        translate(*this, impl->precision, impl->seed, t);
    } catch (Unsupported &e) {
        throw std::runtime_error(std::string("GpuModuleList: ") + e.what());
    }
    std::ostringstream os;
    os << "GpuModuleList plan (" << (impl->precision == CRP_PRECISION_MIXED ? "mixed" : "fp64")
       << ", seed " << impl->seed << ")\n"
       << t.text.str();
    return os.str();
}

std::string GpuModuleList::getDescription() const {
    return "GpuModuleList (device stepping path)\n" + ModuleList::getDescription();
}

void GpuModuleList::run(Candidate *candidate, bool recursive, bool secondariesFirst) {
    candidate_vector_t v(1, ref_ptr<Candidate>(candidate));
    run(&v, recursive, secondariesFirst);
}

void GpuModuleList::run(ref_ptr<Candidate> candidate, bool recursive, bool secondariesFirst) {
    run(candidate.get(), recursive, secondariesFirst);
}

void GpuModuleList::addStats(crp_run_stats &total, uint64_t &events) const {
    total.particle_steps += impl->stats.particle_steps;
    total.tries += impl->stats.tries;
    total.field_evaluations += impl->stats.field_evaluations;
    total.launches += impl->stats.launches;
    total.device_ms += impl->stats.device_ms;
    events += impl->events;
}

// ModuleList::run(candidates) (ModuleList.cpp.in:97-151) in batches: a
// signal stops the batches that have not started; the started one runs to
// completion.  Then, as the reference does: restore the previous handlers,
// raise the signal again, report, and hand the sorted indices of the
// candidates not started to the interrupt action.
void GpuModuleList::run(const candidate_vector_t *candidates, bool recursive,
                        bool secondariesFirst) {
    std::string why;
    if (!isSupported(&why)) {
        if (impl->cpuFallback) {
            ModuleList::run(candidates, recursive, secondariesFirst);
            return;
        }
        throw std::runtime_error("GpuModuleList: chain is not on the device path: " + why);
    }
    const size_t count = candidates->size();
    crp_run_stats total;
    std::memset(&total, 0, sizeof(total));
    uint64_t events = 0;
    std::vector<int> notFinished;
    int signal_seen = 0;
    {
        SignalScope sig;
        for (size_t done = 0; done < count;) {
            const size_t n = std::min(impl->batch, count - done);
            if (g_cancel != 0) {
                for (size_t i = done; i < done + n; i++) notFinished.push_back(int(i));
            } else {
                candidate_vector_t v(candidates->begin() + done, candidates->begin() + done + n);
                runDevice(v);
                addStats(total, events);
            }
            done += n;
        }
        signal_seen = g_cancel;
    }
    impl->stats = total;
    impl->events = events;
    if (signal_seen > 0) {
        raise(signal_seen);
        std::cerr << "############################################################################\n";
        std::cerr << "#\tInterrupted CRPropa simulation \n";
        std::cerr << "# A total of " << notFinished.size() << " candidates have not been started.\n";
        std::cerr << "# the indices of the vector haven been written to to output file. \n";
        std::cerr << "############################################################################\n";
        std::sort(notFinished.begin(), notFinished.end());
        if (this->*member(ListHaveInterruptAction()))
            (this->*member(ListInterruptAction()))->dumpIndexList(notFinished);
    }
}

// ModuleList::run(source, count) (ModuleList.cpp.in:153-214) in batches of
// candidates drawn on this thread; a signal stops the draws, as in the
// reference, which reports the count of candidates not started.
void GpuModuleList::run(SourceInterface *source, size_t count, bool recursive,
                        bool secondariesFirst) {
    std::string why;
    if (!isSupported(&why)) {
        if (impl->cpuFallback) {
            ModuleList::run(source, count, recursive, secondariesFirst);
            return;
        }
        throw std::runtime_error("GpuModuleList: chain is not on the device path: " + why);
    }
    crp_run_stats total;
    std::memset(&total, 0, sizeof(total));
    uint64_t events = 0;
    size_t not_started = 0;
    int signal_seen = 0;
    {
        SignalScope sig;
        for (size_t done = 0; done < count;) {
            size_t n = std::min(impl->batch, count - done);
            if (g_cancel != 0) {
                not_started += n;
            } else {
                candidate_vector_t v;
                v.reserve(n);
                for (size_t i = 0; i < n; i++) v.push_back(source->getCandidate());
                runDevice(v);
                addStats(total, events);
            }
            done += n;
        }
        signal_seen = g_cancel;
    }
    impl->stats = total;
    impl->events = events;
    if (signal_seen > 0) {
        raise(signal_seen);
        std::cerr << "############################################################################\n";
        std::cerr << "# Interrupted CRPropa simulation \n";
        std::cerr << "# Number of not started candidates from source: " << not_started << "\n";
        std::cerr << "############################################################################\n";
    }
}

void GpuModuleList::runDevice(const candidate_vector_t &cands) {
    Translation t;
    translate(*this, impl->precision, impl->seed, t);
    std::memset(&impl->stats, 0, sizeof(impl->stats));
    impl->events = 0;
    const size_t n = cands.size();
    if (n == 0) return;

    // plan: rebuilt when the chain, its parameters or its field payload changed
    if (!impl->plan || impl->planFingerprint != t.fp.h) {
        if (impl->plan) {
            crp_plan_destroy(impl->plan);
            impl->plan = 0;
        }
        crp_plan_desc d;
        std::memset(&d, 0, sizeof(d));
        d.abi_version = CRP_ABI_VERSION;
        d.precision = impl->precision;
        d.fields = &t.fields[0];
        d.n_fields = int32_t(t.fields.size());
        d.modules = &t.modules[0];
        d.n_modules = int32_t(t.modules.size());
        d.seed = impl->seed;
        check(crp_plan_create(&d, &impl->plan));
        impl->planFingerprint = t.fp.h;
        impl->eventsPerCandidate = 0;
    }

    const bool per = !t.perCandidateKey.empty();
    Batch b;
    b.resize(n, per, t.needsStepCount);
    for (size_t i = 0; i < n; i++) {
        const Candidate *c = cands[i].get();
        const ParticleState &s = c->current;
        b.id[i] = s.getId();
        b.charge[i] = s.getCharge();
        b.energy[i] = s.getEnergy();
        const Vector3d &p = s.getPosition(), &u = s.getDirection(),
                       &q = c->previous.getPosition();
        b.x[i] = p.x; b.y[i] = p.y; b.z[i] = p.z;
        b.dx[i] = u.x; b.dy[i] = u.y; b.dz[i] = u.z;
        b.px[i] = q.x; b.py[i] = q.y; b.pz[i] = q.z;
        b.length[i] = c->getTrajectoryLength();
        b.time[i] = c->getTime();
        b.cur[i] = c->getCurrentStep();
        b.next[i] = c->getNextStep();
        b.active[i] = c->isActive() ? 1 : 0;
        b.flags[i] = 0;
        if (per) b.max_length[i] = c->getProperty(t.perCandidateKey).asDouble();
        if (t.needsStepCount) b.steps[i] = 0;
    }

    // every recording module fires at most once per candidate when it
    // deactivates; observers that keep candidates active may fire more often.
    // The capacity also covers the most records per candidate an earlier run
    // of this plan produced; when a run still overflows it, the batch is run
    // again with the exact count (the inputs are intact) and a note says so.
    size_t nrec = 0;
    for (size_t m = 0; m < t.modules.size(); m++) nrec += t.modules[m].record ? 1 : 0;
    Records rec;
    const double per_cand = std::max<double>(double(std::max<size_t>(nrec, 1)), 1.25 * impl->eventsPerCandidate);
    uint64_t cap = uint64_t(double(n) * per_cand) + 1024;
    for (int attempt = 0;; attempt++) {
        Batch work = b;
        crp_candidates view = work.view();
        crp_records rv = rec.view(cap);
        crp_run_opts o;
        std::memset(&o, 0, sizeof(o));
        o.mode = CRP_MODE_AUTO;
        o.records = nrec ? &rv : 0;
        // a started batch runs to completion (no cancel flag): the callers
        // stop between batches
        check(crp_run(impl->plan, &view, n, &o, &impl->stats));
        if (rec.count > cap) {
            if (attempt > 0) throw std::runtime_error("GpuModuleList: record count changed between runs");
            std::cerr << "GpuModuleList: " << rec.count << " detection/reject records overflowed the "
                      << cap << " reserved; running the batch of " << n << " candidates again\n";
            cap = rec.count;
            continue;
        }
        if (n) impl->eventsPerCandidate = std::max(impl->eventsPerCandidate, double(rec.count) / double(n));
        std::swap(b, work);  // keep the results
        break;
    }

    // events per candidate in the order the device wrote them (one thread
    // writes all of a candidate's records, so slot order is time order)
    const uint64_t ne = nrec ? rec.count : 0;
    std::vector<uint64_t> order(ne);
    for (uint64_t e = 0; e < ne; e++) order[e] = e;
    std::stable_sort(order.begin(), order.end(),
                     [&rec](uint64_t a, uint64_t c) { return rec.index[a] < rec.index[c]; });
    impl->events = ne;

    size_t e = 0;
    for (size_t i = 0; i < n; i++) {
        Candidate *c = cands[i].get();
        for (; e < ne && rec.index[order[e]] == i; e++) {
            const uint64_t r = order[e];
            const int mi = rec.module[r];
            if (mi < 0 || size_t(mi) >= t.actions.size())
                throw std::runtime_error("GpuModuleList: record of an unknown module");
            c->current.setPosition(Vector3d(rec.x[r], rec.y[r], rec.z[r]));
            set_direction_exact(c->current, rec.dx[r], rec.dy[r], rec.dz[r]);
            c->setTrajectoryLength(rec.length[r]);
            c->setTime(rec.time[r]);
            const Action &a = t.actions[mi];
            if (a.kind == CRP_MODULE_MAX_TRAJECTORY_LENGTH || a.kind == CRP_MODULE_BOUNDARY) {
                // AbstractCondition::reject (Module.cpp:25-37)
                const ref_ptr<Module> &act = a.condition->*member(RejectAction());
                if (act.valid()) act->process(c);
                const std::string &k = a.condition->*member(RejectKey());
                if (!k.empty()) c->setProperty(k, a.condition->*member(RejectValue()));
            } else if (a.kind == CRP_MODULE_OBSERVER) {
                // Observer::process after a detection (Observer.cpp:37-52)
                const FeatureList &fs = a.observer->*member(ObserverFeatures());
                for (size_t f = 0; f < fs.size(); f++) fs[f]->onDetection(c);
                const ref_ptr<Module> &act = a.observer->*member(ObserverAction());
                if (act.valid()) {
                    if (a.observer->*member(ObserverClone()))
                        act->process(c->clone(false));
                    else
                        act->process(c);
                }
                const std::string &k = a.observer->*member(ObserverFlagKey());
                if (!k.empty()) c->setProperty(k, a.observer->*member(ObserverFlagValue()));
            }
        }
        // final state
        c->current.setPosition(Vector3d(b.x[i], b.y[i], b.z[i]));
        set_direction_exact(c->current, b.dx[i], b.dy[i], b.dz[i]);
        c->previous.setPosition(Vector3d(b.px[i], b.py[i], b.pz[i]));
        c->setCurrentStep(b.cur[i]);  // also adds to length and time: both set next
        c->setTrajectoryLength(b.length[i]);
        c->setTime(b.time[i]);
        c->setNextStep(b.next[i]);
        c->setActive(b.active[i] != 0);
    }
}

}  // namespace crpgpu
