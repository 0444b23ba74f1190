/*
 * ref_shim.cpp -- TEST INFRASTRUCTURE, not product code.
 *
 * Drives the reference's own CPU modules (CRPropa3, compiled from its
 * sources by oracle/Makefile into oracle/_ref/) from the plain arrays of
 * include/crp_gpu.h, so that the tests, the golden-fixture generator and
 * bench.py's CPU baseline can run the unmodified reference path on exactly
 * the inputs the device path gets.  Only tests/, bench.py's reference arm and
 * __graft_entry__.smoke() load this library.
 *
 * What comes from the reference (unchanged, linked): Candidate, ModuleList
 * (src/ModuleList.cpp.in:97 run(candidate_vector) with OpenMP
 * schedule(static,100)), PropagationCK, PropagationBP, DiffusionSDE,
 * MagneticFieldGrid (trilinear, tricubic and nearest-neighbour Grid3f),
 * ModulatedMagneticFieldGrid, JF12Field, PlanckJF12bField, UF23Field,
 * PeriodicMagneticField, MagneticFieldList,
 * UniformMagneticField, PlaneWaveTurbulence, MaximumTrajectoryLength,
 * Observer, ObserverSurface(Sphere), ObserverDetectAll, TextOutput,
 * ParticleCollector, Source
 * features and Random.
 *
 * Helpers written here (no reference counterpart):
 *   ToroidalField         B = b0 (-y, x, 0)/r  (analytic field of the
 *                         diffusion workload; ToroidalHaloField has another
 *                         form)
 *   PerCandidateLength    MaximumTrajectoryLength with the limit read from a
 *                         candidate property (one limit per candidate)
 *   RecordAction          detection / reject action that stores a record
 *   StepCounter           counts process() calls of the chain = steps
 */
#include "crp_gpu.h"
#include "ref_chain.h"

#include "crpropa/Candidate.h"
#include "crpropa/Grid.h"
#include "crpropa/GridTools.h"
#include "crpropa/ModuleList.h"
#include "crpropa/Random.h"
#include "crpropa/Source.h"
#include "crpropa/Units.h"
#include "crpropa/magneticField/MagneticField.h"
#include "crpropa/magneticField/JF12Field.h"
#include "crpropa/magneticField/JF12FieldSolenoidal.h"
#include "crpropa/magneticField/MagneticFieldGrid.h"
#include "crpropa/magneticField/UF23Field.h"
#include "crpropa/magneticField/PT11Field.h"
#include "crpropa/magneticField/TF17Field.h"
#include "crpropa/magneticField/PolarizedSingleModeMagneticField.h"
#include "crpropa/magneticField/KST24Field.h"
#include "crpropa/magneticField/CMZField.h"
#include "crpropa/magneticField/ArchimedeanSpiralField.h"
#include "crpropa/magneticField/turbulentField/PlaneWaveTurbulence.h"
#include "crpropa/magneticField/turbulentField/TurbulentField.h"
#include "crpropa/module/Boundary.h"
#include "crpropa/module/BreakCondition.h"
#include "crpropa/module/DiffusionSDE.h"
#include "crpropa/advectionField/AdvectionField.h"
#include "crpropa/advectionField/TimeDependentAdvectionField.h"
#include "crpropa/module/Observer.h"
#include "crpropa/module/ParticleCollector.h"
#include "crpropa/module/PropagationBP.h"
#include "crpropa/module/PropagationCK.h"
#include "crpropa/module/TextOutput.h"
#include "crpropa/Geometry.h"

#include <dlfcn.h>
#include <omp.h>

#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

using namespace crpropa;

namespace {
std::string g_error;
}

namespace crp_ref {

/* The mass table is read on the first ParticleState::setId of a nucleus
 * (ParticleMass.cpp:24); the stepping path never uses the mass.  Point
 * CRPROPA_DATA_PATH at the stub table the Makefile writes beside this
 * library. */
void ensure_data_path() {
    static bool done = false;
    if (done) return;
    done = true;
    Dl_info info;
    if (dladdr((void *)&ensure_data_path, &info) && info.dli_fname) {
        std::string p(info.dli_fname);
        size_t s = p.rfind('/');
        std::string dir = (s == std::string::npos) ? std::string(".") : p.substr(0, s);
        setenv("CRPROPA_DATA_PATH", (dir + "/data").c_str(), 1);
    }
}

class ToroidalField : public MagneticField {
    double b0;
public:
    explicit ToroidalField(double b0) : b0(b0) {}
    Vector3d getField(const Vector3d &p) const {
        double r = std::sqrt(p.x * p.x + p.y * p.y);
        return Vector3d(-p.y, p.x, 0.) * (b0 / r);
    }
};

class PerCandidateLength : public AbstractCondition {
public:
    void process(Candidate *c) const {
        double maxLength = c->getProperty("CrpMaxLength").asDouble();
        double length = c->getTrajectoryLength();
        if (length >= maxLength)
            reject(c);
        else
            c->limitNextStep(maxLength - length);
    }
};

class RecordAction : public Module {
    crp_records *rec;
    int module;
public:
    RecordAction(crp_records *rec, int module) : rec(rec), module(module) {}
    void process(Candidate *c) const {
        if (!rec) return;
        uint64_t slot;
#pragma omp critical(crp_record)
        { slot = (*rec->count)++; }
        if (slot >= rec->capacity) return;
        rec->index[slot] = (uint64_t)c->getProperty("CrpIndex").asUInt64();
        rec->module[slot] = module;
        rec->trajectory_length[slot] = c->getTrajectoryLength();
        rec->time[slot] = c->getTime();
        const Vector3d &p = c->current.getPosition();
        const Vector3d &d = c->current.getDirection();
        rec->x[slot] = p.x; rec->y[slot] = p.y; rec->z[slot] = p.z;
        rec->dx[slot] = d.x; rec->dy[slot] = d.y; rec->dz[slot] = d.z;
        rec->energy[slot] = c->current.getEnergy();
        rec->id[slot] = c->current.getId();
    }
};

StepCounter::StepCounter() : perThread(256 * 8, 0) {}
void StepCounter::process(Candidate *c) const { perThread[omp_get_thread_num() * 8]++; }
uint64_t StepCounter::total() const {
    uint64_t s = 0;
    for (size_t i = 0; i < perThread.size(); i += 8) s += perThread[i];
    return s;
}

// A Grid3f (width 3) or Grid1f (width 1) holding a crp_grid3f_desc's values,
// boundary flags and interpolation type.
template <typename T>
static ref_ptr<Grid<T> > make_grid(const crp_grid3f_desc &g, int width, Built &b) {
    ref_ptr<Grid<T> > grid = new Grid<T>(Vector3d(g.origin[0], g.origin[1], g.origin[2]), g.nx, g.ny,
                                         g.nz, Vector3d(g.spacing[0], g.spacing[1], g.spacing[2]));
    grid->setReflective(g.reflective != 0);
    grid->setClipVolume(g.clip_volume != 0);
    grid->setInterpolationType((interpolationType)g.interpolation);
    std::vector<T> &v = grid->getGrid();
    std::memcpy(&v[0], g.values, sizeof(float) * width * g.nx * g.ny * g.nz);
    b.keep.push_back(grid.get());
    return grid;
}

static ref_ptr<MagneticField> build_component(const crp_field_component &f, Built &b,
                                              const Helpers *h) {
    ref_ptr<MagneticField> m;
    if (f.kind == CRP_FIELD_GRID) {
        m = new MagneticFieldGrid(make_grid<Vector3f>(f.grid, 3, b));
    } else if (f.kind == CRP_FIELD_MODULATED_GRID) {
        ref_ptr<Grid3f> grid = make_grid<Vector3f>(f.grid, 3, b);
        ref_ptr<Grid1f> mod = make_grid<float>(f.modulation, 1, b);
        ref_ptr<ModulatedMagneticFieldGrid> mm = new ModulatedMagneticFieldGrid(grid, mod);
        // the constructor resets both flags (MagneticFieldGrid.cpp:22-23)
        mm->setReflective(f.grid.reflective != 0, f.modulation.reflective != 0);
        m = mm;
    } else if (f.kind == CRP_FIELD_JF12) {
        // the constructors set the parameters (JF12Field.cpp:8, :352); the
        // descriptor's flags and grids go through the public setters
        const crp_jf12_desc &j = f.jf12;
        if (j.kpc == 0) throw std::runtime_error("ref_shim: JF12 parameters not set");
        ref_ptr<JF12Field> jf;
        if (j.variant == CRP_JF12_SOLENOIDAL) {  // JF12FieldSolenoidal(delta, zs) and its setters
            JF12FieldSolenoidal *s = new JF12FieldSolenoidal(j.delta, j.z_s);
            if (j.r2s == j.r2) s->deactivateOuterTransition();
            jf = s;
        } else if (j.variant == CRP_JF12_PLANCK) {
            jf = new PlanckJF12bField();
        } else {
            jf = new JF12Field();
        }
        jf->setUseRegularField(j.use_regular != 0);
        jf->setUseDiskField(j.use_disk != 0);
        jf->setUseToroidalHaloField(j.use_toroidal_halo != 0);
        jf->setUseXField(j.use_x != 0);
        if (f.modulation.values) jf->setStriatedGrid(make_grid<float>(f.modulation, 1, b));
        if (f.grid.values) jf->setTurbulentGrid(make_grid<Vector3f>(f.grid, 3, b));
        jf->setUseStriatedField(j.use_striated != 0);
        jf->setUseTurbulentField(j.use_turbulent != 0);
        m = jf;
    } else if (f.kind == CRP_FIELD_UF23) {
        m = new UF23Field((UF23Field::ModelType)f.uf23.model);
    } else if (f.kind == CRP_FIELD_PT11) {  // PT11Field() and the setters that give the switches
        PT11Field *t = new PT11Field();
        if (f.pt11.use_bss) t->setUseBSS(true);
        else if (!f.pt11.use_ass) t->setUseASS(false);
        if (!f.pt11.use_halo) t->setUseHalo(false);
        m = t;
    } else if (f.kind == CRP_FIELD_TF17) {  // TF17Field(disk, halo) and its switches
        TF17Field *t = new TF17Field((TF17DiskModel)f.tf17.disk_model, (TF17HaloModel)f.tf17.halo_model);
        t->setUseDiskField(f.tf17.use_disk != 0);
        t->setUseHaloField(f.tf17.use_halo != 0);
        m = t;
    } else if (f.kind == CRP_FIELD_SINGLE_MODE) {  // the constructor with the original arguments
        const crp_single_mode_desc &s = f.single_mode;
        static const char *ar[] = {"amplitude", "rms"}, *ph[] = {"polarization", "helicity"},
                          *md[] = {"elliptical", "circular", "linear"};
        m = new PolarizedSingleModeMagneticField(
            s.b0, s.wavelength, s.sigma, Vector3d(s.r0[0], s.r0[1], s.r0[2]), Vector3d(s.e1[0], s.e1[1], s.e1[2]),
            Vector3d(s.e2[0], s.e2[1], s.e2[2]), ar[s.amplitude_rms], ph[s.polarization_helicity], md[s.mode]);
    } else if (f.kind == CRP_FIELD_KST24) {  // no parameters
        m = new KST24Field();
    } else if (f.kind == CRP_FIELD_CMZ) {  // CMZField() and its four switches
        CMZField *c = new CMZField();
        c->setUseMCField(f.cmz.use_mc != 0);
        c->setUseICField(f.cmz.use_ic != 0);
        c->setUseNTFField(f.cmz.use_ntf != 0);
        c->setUseRadioArc(f.cmz.use_radio_arc != 0);
        m = c;
    } else if (f.kind == CRP_FIELD_ARCHIMEDEAN_SPIRAL) {
        const crp_archimedean_desc &a = f.archimedean;
        m = new ArchimedeanSpiralField(a.b0, a.r0, a.omega, a.vw);
    } else if (f.kind == CRP_FIELD_PLANE_WAVE) {
        const crp_plane_wave_desc &p = f.plane_wave;
        TurbulenceSpectrum *spec = new TurbulenceSpectrum(p.brms, p.lmin, p.lmax, p.lbendover,
                                                          p.sindex, p.qindex);
        b.keep.push_back(spec);
        m = new PlaneWaveTurbulence(*spec, p.n_modes, p.seed);
    } else if (f.kind == CRP_FIELD_UNIFORM) {
        m = new UniformMagneticField(Vector3d(f.uniform[0], f.uniform[1], f.uniform[2]));
    } else if (f.kind == CRP_FIELD_TOROIDAL) {
        m = h ? h->toroidal(f.toroidal_b0) : new ToroidalField(f.toroidal_b0);
    } else {
        throw std::runtime_error("ref_shim: unknown field kind");
    }
    if (f.periodic) {
        m = new PeriodicMagneticField(
            m, Vector3d(f.periodic_extends[0], f.periodic_extends[1], f.periodic_extends[2]),
            Vector3d(f.periodic_origin[0], f.periodic_origin[1], f.periodic_origin[2]),
            f.periodic_reflective != 0);
    }
    return m;
}

static ref_ptr<MagneticField> build_field(const crp_plan_desc *d, Built &b, const Helpers *h) {
    if (d->n_fields == 1)
        return build_component(d->fields[0], b, h);
    ref_ptr<MagneticFieldList> list = new MagneticFieldList();
    for (int i = 0; i < d->n_fields; i++)
        list->addField(build_component(d->fields[i], b, h));
    return list;
}

// The reference's observer feature for a crp_observer_feature_desc.
static ObserverFeature *build_feature(const crp_observer_feature_desc &f) {
    const Vector3d a(f.a[0], f.a[1], f.a[2]), bv(f.b[0], f.b[1], f.b[2]);
    switch (f.kind) {
    case CRP_OBSERVER_SURFACE_SPHERE: return new ObserverSurface(new Sphere(a, f.r));
    case CRP_OBSERVER_DETECT_ALL: return new ObserverDetectAll();
    case CRP_OBSERVER_SURFACE_PLANE: return new ObserverSurface(new Plane(a, bv));
    case CRP_OBSERVER_SURFACE_BOX: return new ObserverSurface(new ParaxialBox(a, bv));
    case CRP_OBSERVER_TRACKING: return new ObserverTracking(a, f.r, f.step);
    case CRP_OBSERVER_1D: return new Observer1D();
    case CRP_OBSERVER_INACTIVE_VETO: return new ObserverInactiveVeto();
    case CRP_OBSERVER_NUCLEUS_VETO: return new ObserverNucleusVeto();
    case CRP_OBSERVER_NEUTRINO_VETO: return new ObserverNeutrinoVeto();
    case CRP_OBSERVER_PHOTON_VETO: return new ObserverPhotonVeto();
    case CRP_OBSERVER_ELECTRON_VETO: return new ObserverElectronVeto();
    case CRP_OBSERVER_PARTICLE_ID_VETO: return new ObserverParticleIdVeto(f.particle_id);
    }
    throw std::runtime_error("ref_shim: unknown observer feature");
}

void build_chain(const crp_plan_desc *d, crp_records *rec, Built &b, const Helpers *h,
                 ModuleList *sim, bool count_steps, const char *text_output, int text_type) {
    b.field = build_field(d, b, h);
    b.sim = sim ? sim : new ModuleList();
    for (int i = 0; i < d->n_modules; i++) {
        const crp_module_desc &m = d->modules[i];
        if (m.kind == CRP_MODULE_PROPAGATION) {
            if (m.propagator == CRP_PROP_CK) {
                b.sim->add(new PropagationCK(b.field, m.tolerance, m.min_step, m.max_step));
            } else if (m.propagator == CRP_PROP_BP) {
                if (m.min_step == m.max_step)
                    b.sim->add(new PropagationBP(b.field, m.max_step));
                else
                    b.sim->add(new PropagationBP(b.field, m.tolerance, m.min_step, m.max_step));
            } else if (m.propagator == CRP_PROP_SDE) {
                DiffusionSDE *sde = new DiffusionSDE(b.field, m.tolerance, m.min_step, m.max_step,
                                                     m.sde_epsilon);
                sde->setAlpha(m.sde_alpha);
                sde->setScale(m.sde_scale);
                if (m.n_advection > 0) {  // the advection fields' constructors and setters
                    std::vector<ref_ptr<AdvectionField> > fs;
                    for (int a = 0; a < m.n_advection; a++) {
                        const crp_advection_desc &A = m.advection[a];
                        const Vector3d o(A.origin[0], A.origin[1], A.origin[2]);
                        AdvectionField *f = nullptr;
                        switch (A.kind) {
                        case CRP_ADVECTION_UNIFORM:
                            f = new UniformAdvectionField(Vector3d(A.value[0], A.value[1], A.value[2])); break;
                        case CRP_ADVECTION_CONSTANT_SPHERICAL: f = new ConstantSphericalAdvectionField(o, A.v); break;
                        case CRP_ADVECTION_SPHERICAL:
                            f = new SphericalAdvectionField(o, A.radius, A.v, A.tau, A.alpha); break;
                        case CRP_ADVECTION_CARTESIAN_SHOCK:
                            f = new OneDimensionalCartesianShock(A.compression, A.v, A.length); break;
                        case CRP_ADVECTION_SPHERICAL_SHOCK_1D:
                            f = new OneDimensionalSphericalShock(A.radius, A.v, A.compression, A.length,
                                                                 A.cool_upstream != 0);
                            break;
                        case CRP_ADVECTION_OBLIQUE_SHOCK:
                            f = new ObliqueAdvectionShock(A.compression, A.v, A.vy, A.length); break;
                        case CRP_ADVECTION_SPHERICAL_SHOCK: {
                            SphericalAdvectionShock *s = new SphericalAdvectionShock(o, A.radius, A.v, A.length);
                            s->setRRot(A.r_rot);
                            s->setAzimuthalSpeed(A.v_phi);
                            f = s;
                            break;
                        }
                        case CRP_ADVECTION_TIME_SHOCK: {
                            OneDimensionalTimeDependentShock *s =
                                new OneDimensionalTimeDependentShock(A.v, A.v1, A.v0, A.length);
                            s->setShockPosition(A.x0);
                            s->setShockTime(A.t0);
                            f = s;
                            break;
                        }
                        case CRP_ADVECTION_SEDOV_TAYLOR:
                            f = new SedovTaylorBlastWave(A.energy, A.density, A.length); break;
                        default: throw std::runtime_error("ref_shim: unknown advection field");
                        }
                        fs.push_back(f);
                    }
                    if (fs.size() == 1) {
                        sde->setAdvectionField(fs[0]);
                    } else {
                        AdvectionFieldList *l = new AdvectionFieldList();
                        for (auto &f : fs) l->addField(f);
                        sde->setAdvectionField(l);
                    }
                }
                b.sim->add(sde);
            } else {
                throw std::runtime_error("ref_shim: unknown propagator");
            }
        } else if (m.kind == CRP_MODULE_MAX_TRAJECTORY_LENGTH) {
            AbstractCondition *c;
            if (m.per_candidate_length)
                c = h ? h->perCandidateLength() : new PerCandidateLength();
            else
                c = new MaximumTrajectoryLength(m.max_length);
            if (m.record) c->onReject(new RecordAction(rec, i));
            b.sim->add(c);
        } else if (m.kind == CRP_MODULE_OBSERVER) {
            Observer *o = new Observer();
            if (m.n_features == 0) {
                if (m.observer_feature == CRP_OBSERVER_SURFACE_SPHERE)
                    o->add(new ObserverSurface(new Sphere(
                        Vector3d(m.sphere_center[0], m.sphere_center[1], m.sphere_center[2]),
                        m.sphere_radius)));
                else
                    o->add(new ObserverDetectAll());
            }
            for (int f = 0; f < m.n_features; f++) o->add(build_feature(m.features[f]));
            o->setDeactivateOnDetection(m.deactivate_on_detection != 0);
            o->setFlag("Detected", "Detected");
            if (text_output && text_type == kCollectorOutput) {
                ref_ptr<ParticleCollector> pc = new ParticleCollector();
                pc->setClone(true);
                o->onDetection(pc);
                b.collectors.push_back(pc.get());
                b.collector_path = text_output;
            } else if (text_output)
                o->onDetection(new TextOutput(text_output, (Output::OutputType)text_type));
            else if (m.record)
                o->onDetection(new RecordAction(rec, i));
            b.sim->add(o);
        } else if (m.kind == CRP_MODULE_BOUNDARY) {
            const Vector3d a(m.boundary_a[0], m.boundary_a[1], m.boundary_a[2]);
            AbstractCondition *c;
            if (m.boundary == CRP_BOUNDARY_SPHERICAL) {
                SphericalBoundary *bnd = new SphericalBoundary(a, m.boundary_size);
                bnd->setMargin(m.boundary_margin);
                bnd->setLimitStep(m.boundary_limit_step != 0);
                c = bnd;
            } else if (m.boundary == CRP_BOUNDARY_CUBIC) {
                CubicBoundary *bnd = new CubicBoundary(a, m.boundary_size);
                bnd->setMargin(m.boundary_margin);
                bnd->setLimitStep(m.boundary_limit_step != 0);
                c = bnd;
            } else if (m.boundary == CRP_BOUNDARY_ELLIPSOIDAL) {
                EllipsoidalBoundary *bnd = new EllipsoidalBoundary(
                    a, Vector3d(m.boundary_b[0], m.boundary_b[1], m.boundary_b[2]), m.boundary_size);
                bnd->setMargin(m.boundary_margin);
                bnd->setLimitStep(m.boundary_limit_step != 0);
                c = bnd;
            } else {
                CylindricalBoundary *bnd = new CylindricalBoundary(a, m.boundary_size, m.boundary_radius);
                bnd->setMargin(m.boundary_margin);
                bnd->setLimitStep(m.boundary_limit_step != 0);
                c = bnd;
            }
            if (m.record) c->onReject(new RecordAction(rec, i));
            b.sim->add(c);
        } else {
            throw std::runtime_error("ref_shim: unknown module kind");
        }
    }
    if (count_steps) {
        b.counter = new StepCounter();
        b.sim->add(b.counter.get());
    }
}

void load_candidates(const crp_candidates *c, uint64_t n, ModuleList::candidate_vector_t &cands) {
    cands.clear();
    cands.reserve(n);
    for (uint64_t i = 0; i < n; i++) {
        ref_ptr<Candidate> cand = new Candidate(
            c->id[i], c->energy[i], Vector3d(c->x[i], c->y[i], c->z[i]),
            Vector3d(c->dx[i], c->dy[i], c->dz[i]));
        cand->previous.setPosition(Vector3d(c->px[i], c->py[i], c->pz[i]));
        cand->setTrajectoryLength(c->trajectory_length[i]);
        cand->setTime(c->time[i]);
        cand->setNextStep(c->next_step[i]);
        cand->setActive(c->active[i] != 0);
        cand->setProperty("CrpIndex", Variant((uint64_t)i));
        if (c->max_length)
            cand->setProperty("CrpMaxLength", Variant(c->max_length[i]));
        cands.push_back(cand);
    }
}

void store_candidates(const ModuleList::candidate_vector_t &cands, const crp_candidates *c) {
    for (uint64_t i = 0; i < cands.size(); i++) {
        Candidate *cand = cands[i];
        const Vector3d &p = cand->current.getPosition();
        const Vector3d &d = cand->current.getDirection();
        const Vector3d &q = cand->previous.getPosition();
        c->x[i] = p.x; c->y[i] = p.y; c->z[i] = p.z;
        c->dx[i] = d.x; c->dy[i] = d.y; c->dz[i] = d.z;
        c->px[i] = q.x; c->py[i] = q.y; c->pz[i] = q.z;
        c->trajectory_length[i] = cand->getTrajectoryLength();
        c->time[i] = cand->getTime();
        c->current_step[i] = cand->getCurrentStep();
        c->next_step[i] = cand->getNextStep();
        c->active[i] = cand->isActive() ? 1 : 0;
        uint32_t fl = 0;
        if (cand->hasProperty("Rejected")) fl |= CRP_FLAG_REJECTED;
        if (cand->hasProperty("Detected")) fl |= CRP_FLAG_DETECTED;
        c->flags[i] = fl;
    }
}

void finish_outputs(Built &b) {
    if (b.collectors.empty()) return;
    ParticleCollector *pc = dynamic_cast<ParticleCollector *>(b.collectors[0].get());
    if (pc) pc->dump(b.collector_path);
}

}  // namespace crp_ref

using namespace crp_ref;

extern "C" {

const char *ref_last_error() { return g_error.c_str(); }

/* Run the reference ModuleList over n candidates given as arrays (in/out).
 * nthreads OpenMP threads; Random::seedThreads(seed) before the run.
 * Returns 0 on success, and the number of chain process() calls (= steps
 * taken, one per candidate per loop iteration) in *steps. */
int ref_run(const crp_plan_desc *desc, const crp_candidates *c, uint64_t n,
            crp_records *rec, int nthreads, uint32_t seed, uint64_t *steps,
            double *seconds) {
    try {
        ensure_data_path();
        Built b;
        build_chain(desc, rec, b, 0, 0, true, 0, 0);
        ModuleList::candidate_vector_t cands;
        load_candidates(c, n, cands);
        if (nthreads > 0) omp_set_num_threads(nthreads);
        Random::seedThreads(seed);
        // ModuleList::run prints a thread-count banner on stdout; keep
        // stdout clean for the caller.
        std::streambuf *old = std::cout.rdbuf();
        std::ostringstream sink;
        std::cout.rdbuf(sink.rdbuf());
        double t0 = omp_get_wtime();
        b.sim->run(&cands, true, false);
        double t1 = omp_get_wtime();
        std::cout.rdbuf(old);
        if (seconds) *seconds = t1 - t0;
        if (steps) *steps = b.counter->total();
        store_candidates(cands, c);
        return 0;
    } catch (std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

/* The same run with a TextOutput(path, output_type) as every observer's
 * detection action (Observer::onDetection, Observer.cpp:22) instead of the
 * record action; serial numbers start at serial0 (Candidate.h:170). */
int ref_run_textout(const crp_plan_desc *desc, const crp_candidates *c, uint64_t n,
                    const char *path, int output_type, int nthreads, uint32_t seed,
                    uint64_t serial0) {
    try {
        ensure_data_path();
        Built b;
        {
            build_chain(desc, 0, b, 0, 0, false, path, output_type);
            Candidate::setNextSerialNumber(serial0);
            ModuleList::candidate_vector_t cands;
            load_candidates(c, n, cands);
            if (nthreads > 0) omp_set_num_threads(nthreads);
            Random::seedThreads(seed);
            std::streambuf *old = std::cout.rdbuf();
            std::ostringstream sink;
            std::cout.rdbuf(sink.rdbuf());
            b.sim->run(&cands, true, false);
            std::cout.rdbuf(old);
            store_candidates(cands, c);
        }
        finish_outputs(b);
        b.sim = 0;  // closes the TextOutput files
        return 0;
    } catch (std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

/* Field of the chain description at n positions (planar xyz in/out). */
int ref_field_eval(const crp_plan_desc *desc, uint64_t n, const double *pos, double *out) {
    try {
        ensure_data_path();
        Built b;
        ref_ptr<MagneticField> f = build_field(desc, b, 0);
        for (uint64_t i = 0; i < n; i++) {
            Vector3d B = f->getField(Vector3d(pos[i], pos[n + i], pos[2 * n + i]));
            out[i] = B.x; out[n + i] = B.y; out[2 * n + i] = B.z;
        }
        return 0;
    } catch (std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

/* Draw `n` values from crpropa::Random seeded with `seed`:
 * kind 0 rand(), 1 randUniform(a,b), 2 randVector() (3 per draw),
 * 3 randPowerLaw(a, b, c) with index a, 4 randNorm(), 5 randConeVector around
 * (0,0,1) with angle a (3 per draw), 6 randInt() */
int ref_random(uint32_t seed, int kind, uint64_t n, double a, double b, double c, double *out) {
    Random r(seed);
    for (uint64_t i = 0; i < n; i++) {
        switch (kind) {
        case 0: out[i] = r.rand(); break;
        case 1: out[i] = r.randUniform(a, b); break;
        case 2: { Vector3d v = r.randVector(); out[3*i] = v.x; out[3*i+1] = v.y; out[3*i+2] = v.z; } break;
        case 3: out[i] = r.randPowerLaw(a, b, c); break;
        case 4: out[i] = r.randNorm(); break;
        case 5: { Vector3d v = r.randConeVector(Vector3d(0, 0, 1), a); out[3*i] = v.x; out[3*i+1] = v.y; out[3*i+2] = v.z; } break;
        case 6: out[i] = (double)r.randInt(); break;
        default: g_error = "ref_random: unknown kind"; return 1;
        }
    }
    return 0;
}

/* The reference's grid files (GridTools.cpp:134-482): dumpGrid /
 * dumpGridToTxt of a Grid3f (width 3) or Grid1f (width 1) holding `values`,
 * and loadGrid / loadGridFromTxt into one of the given shape. */
static crp_grid3f_desc io_desc(const float *values, uint64_t nx, uint64_t ny, uint64_t nz, const double *origin,
                               const double *spacing, int reflective, int clip, int interp) {
    crp_grid3f_desc g;
    std::memset(&g, 0, sizeof(g));
    g.values = values;
    g.nx = nx; g.ny = ny; g.nz = nz;
    for (int a = 0; a < 3; a++) {
        g.origin[a] = origin ? origin[a] : 0.0;
        g.spacing[a] = spacing ? spacing[a] : 1.0;
    }
    g.reflective = reflective;
    g.clip_volume = clip;
    g.interpolation = interp;
    return g;
}

int ref_dump_grid(const float *values, int width, uint64_t nx, uint64_t ny, uint64_t nz, const char *path,
                  double c, int txt, int save_prop, const double *origin, const double *spacing, int reflective,
                  int clip, int interp) {
    try {
        Built b;
        crp_grid3f_desc g = io_desc(values, nx, ny, nz, origin, spacing, reflective, clip, interp);
        if (width == 3) {
            ref_ptr<Grid3f> grid = make_grid<Vector3f>(g, 3, b);
            if (txt) dumpGridToTxt(grid, path, c, save_prop != 0);
            else dumpGrid(grid, path, c);
        } else {
            ref_ptr<Grid1f> grid = make_grid<float>(g, 1, b);
            if (txt) dumpGridToTxt(grid, path, c, save_prop != 0);
            else dumpGrid(grid, path, c);
        }
        return 0;
    } catch (std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

int ref_load_grid(float *values, int width, uint64_t nx, uint64_t ny, uint64_t nz, const char *path, double c,
                  int txt) {
    try {
        size_t cells = nx * ny * nz;
        if (width == 3) {
            ref_ptr<Grid3f> grid = new Grid3f(Vector3d(0.), nx, ny, nz, Vector3d(1.));
            if (txt) loadGridFromTxt(grid, path, c);
            else loadGrid(grid, path, c);
            std::memcpy(values, &grid->getGrid()[0], sizeof(float) * 3 * cells);
        } else {
            ref_ptr<Grid1f> grid = new Grid1f(Vector3d(0.), nx, ny, nz, Vector3d(1.));
            if (txt) loadGridFromTxt(grid, path, c);
            else loadGrid(grid, path, c);
            std::memcpy(values, &grid->getGrid()[0], sizeof(float) * cells);
        }
        return 0;
    } catch (std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

/* loadGrid3fFromTxt / loadGrid1fFromTxt (GridTools.cpp:262, :354): the
 * properties read from the header (shape, origin, spacing, flags), and the
 * values into `values` if it is large enough (capacity in floats). */
int ref_load_grid_props(const char *path, int width, double c, uint64_t *shape, double *origin, double *spacing,
                        int *flags, float *values, uint64_t capacity) {
    try {
        if (width == 3) {
            ref_ptr<Grid3f> g = loadGrid3fFromTxt(path, c);
            shape[0] = g->getNx(); shape[1] = g->getNy(); shape[2] = g->getNz();
            for (int a = 0; a < 3; a++) { origin[a] = g->getOrigin().data[a]; spacing[a] = g->getSpacing().data[a]; }
            flags[0] = g->isReflective(); flags[1] = g->getClipVolume(); flags[2] = g->getInterpolationType();
            size_t n = 3 * g->getGrid().size();
            if (n <= capacity) std::memcpy(values, &g->getGrid()[0], sizeof(float) * n);
        } else {
            ref_ptr<Grid1f> g = loadGrid1fFromTxt(path, c);
            shape[0] = g->getNx(); shape[1] = g->getNy(); shape[2] = g->getNz();
            for (int a = 0; a < 3; a++) { origin[a] = g->getOrigin().data[a]; spacing[a] = g->getSpacing().data[a]; }
            flags[0] = g->isReflective(); flags[1] = g->getClipVolume(); flags[2] = g->getInterpolationType();
            size_t n = g->getGrid().size();
            if (n <= capacity) std::memcpy(values, &g->getGrid()[0], sizeof(float) * n);
        }
        return 0;
    } catch (std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

/* The draws of the turbulence k-space loops from crpropa::Random seeded
 * with `seed`, for n modes: kind 0 (GridTurbulence.cpp:97, :104) rand,
 * rand; kind 1 (SimpleGridTurbulence.cpp:88-93) rand, randNorm, rand; kind 2
 * (HelicalGridTurbulence.cpp:88-92) randNorm, rand, rand. */
int ref_turbulence_draws(uint32_t seed, int kind, uint64_t n, double *out) {
    Random r;
    r.seed(seed);
    for (uint64_t i = 0; i < n; i++) {
        if (kind == 0) {
            out[2 * i] = r.rand();
            out[2 * i + 1] = r.rand();
        } else if (kind == 1) {
            out[3 * i] = r.rand();
            out[3 * i + 1] = r.randNorm();
            out[3 * i + 2] = r.rand();
        } else {
            out[3 * i] = r.randNorm();
            out[3 * i + 1] = r.rand();
            out[3 * i + 2] = r.rand();
        }
    }
    return 0;
}

/* The striated grid of JF12Field::randomStriated(seed) (JF12Field.cpp:86):
 * 100^3 floats in cell order. */
int ref_jf12_random_striated(int seed, float *out) {
    ref_ptr<JF12Field> jf = new JF12Field();
    jf->randomStriated(seed);
    std::vector<float> &v = jf->getStriatedGrid()->getGrid();
    std::memcpy(out, &v[0], sizeof(float) * v.size());
    return 0;
}

/* Candidates from the reference Source with the features of the stepping
 * workloads: SourcePosition(pos), one or several particle types,
 * SourcePowerLawSpectrum(emin, emax, index), SourceIsotropicEmission, drawn
 * by one thread from Random::seedThreads(seed).  Feature order as added
 * here: position, type(s), spectrum, direction. */
int ref_sample_source(uint32_t seed, uint64_t n, const double *pos, int ntypes,
                      const int32_t *ids, const double *abundances, double emin,
                      double emax, double index, int32_t *id_out, double *e_out,
                      double *dir_out) {
    try {
        ensure_data_path();
        Source src;
        src.add(new SourcePosition(Vector3d(pos[0], pos[1], pos[2])));
        if (ntypes == 1) {
            src.add(new SourceParticleType(ids[0]));
        } else {
            SourceMultipleParticleTypes *m = new SourceMultipleParticleTypes();
            for (int i = 0; i < ntypes; i++) m->add(ids[i], abundances[i]);
            src.add(m);
        }
        src.add(new SourcePowerLawSpectrum(emin, emax, index));
        src.add(new SourceIsotropicEmission());
        omp_set_num_threads(1);
        Random::seedThreads(seed);
        for (uint64_t i = 0; i < n; i++) {
            ref_ptr<Candidate> c = src.getCandidate();
            id_out[i] = c->current.getId();
            e_out[i] = c->current.getEnergy();
            const Vector3d &d = c->current.getDirection();
            dir_out[3*i] = d.x; dir_out[3*i+1] = d.y; dir_out[3*i+2] = d.z;
        }
        return 0;
    } catch (std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

/* Charge the reference assigns to a particle id (ParticleState::setId). */
double ref_charge(int32_t id) {
    ensure_data_path();
    ParticleState s;
    s.setId(id);
    return s.getCharge();
}

/* Write TextOutput(Event3D or Trajectory3D) lines for n candidate states
 * with the reference's own TextOutput into `path` (header included).
 * Source state columns use the src_* arrays. */
int ref_text_output(const char *path, int output_type, uint64_t n, const uint64_t *serial,
                    const int32_t *id, const double *energy, const double *xyz,
                    const double *dir, const double *trajectory_length,
                    const int32_t *src_id, const double *src_energy, const double *src_xyz,
                    const double *src_dir) {
    try {
        ensure_data_path();
        ref_ptr<TextOutput> out = new TextOutput(std::string(path),
                                                 (Output::OutputType)output_type);
        for (uint64_t i = 0; i < n; i++) {
            ref_ptr<Candidate> c = new Candidate(src_id[i], src_energy[i],
                Vector3d(src_xyz[3*i], src_xyz[3*i+1], src_xyz[3*i+2]),
                Vector3d(src_dir[3*i], src_dir[3*i+1], src_dir[3*i+2]));
            c->current.setId(id[i]);
            c->current.setEnergy(energy[i]);
            c->current.setPosition(Vector3d(xyz[3*i], xyz[3*i+1], xyz[3*i+2]));
            c->current.setDirection(Vector3d(dir[3*i], dir[3*i+1], dir[3*i+2]));
            c->setTrajectoryLength(trajectory_length[i]);
            c->setSerialNumber(serial[i]);
            out->process(c);
        }
        out->close();
        return 0;
    } catch (std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

}  // extern "C"
