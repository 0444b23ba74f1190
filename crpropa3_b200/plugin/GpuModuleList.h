// GpuModuleList.h -- CRPropa plugin: a ModuleList whose run() steps the
// chain on a B200 through the engine's C-ABI (crp_gpu.h).
//
// Drop-in for crpropa::ModuleList (include/crpropa/ModuleList.h:24) on
// chains of the charged-particle stepping path:
//
//   propagation   PropagationBP (fixed or adaptive), PropagationCK,
//                 DiffusionSDE (no advection field)
//   fields        MagneticFieldGrid over a Grid3f (trilinear, tricubic or
//                 nearest-neighbour), ModulatedMagneticFieldGrid,
//                 JF12Field and PlanckJF12bField (regular, striated and
//                 turbulent parts), UF23Field (all eight models), PT11Field,
//                 ArchimedeanSpiralField,
//                 PeriodicMagneticField, MagneticFieldList,
//                 UniformMagneticField, PlaneWaveTurbulence,
//                 ToroidalMagneticField (below)
//   conditions    MaximumTrajectoryLength (no observer positions),
//                 CandidateMaximumTrajectoryLength (below),
//                 SphericalBoundary, CubicBoundary, EllipsoidalBoundary,
//                 CylindricalBoundary
//   observers     Observer with up to four features: ObserverSurface over a
//                 Sphere, Plane or ParaxialBox, ObserverDetectAll,
//                 ObserverTracking, Observer1D and the particle vetoes;
//                 any detection action
//
// The user's chain objects are read, not replaced: the same ModuleList code
// that builds a CPU simulation builds this one.  run() packs the candidates
// into structure-of-arrays, runs them to completion on the device and writes
// the state back into the same Candidate objects.  Detection and reject
// actions (TextOutput, Output, ParticleCollector, ...) are the user's own
// modules: the device records each event with the candidate's state at that
// moment, and the plugin calls the action's process() on the host with that
// state, in candidate order, then sets the flag properties the reference
// sets (Observer.cpp:37-52, Module.cpp:25-37).
//
// A chain with any other module or field is not run on the CPU behind the
// caller's back: run() throws std::runtime_error naming the module, unless
// setCpuFallback(true) was called, in which case ModuleList::run runs it.
//
// Differences from ModuleList::run that a caller can see:
//   * Candidate::previous gets the previous position only (the device keeps
//     no previous direction); observers and outputs read no more.
//   * Actions run after the stepping, one candidate after another, instead
//     of inside the OpenMP loop: output line order is by candidate, not by
//     thread timing.
//   * run(source, count) draws candidates on the calling thread, in batches;
//     run(candidates) also runs in batches of setBatchSize().
//   * SIGINT / SIGTERM during a run (ModuleList.cpp.in:110-150): a batch
//     that has started runs to completion, as a started candidate does in
//     the reference; the candidates of the batches not yet started are left
//     unchanged and their indices go, sorted, to the interrupt action's
//     dumpIndexList (run(candidates) with setInterruptAction, as in the
//     reference); then the previous handlers are restored and the signal is
//     raised again.  A started candidate of the reference is one candidate
//     per thread; here it is a whole batch.
//   * Secondaries: the supported modules create none.
#ifndef CRPGPU_GPU_MODULE_LIST_H
#define CRPGPU_GPU_MODULE_LIST_H

#include "crpropa/Candidate.h"
#include "crpropa/Module.h"
#include "crpropa/ModuleList.h"
#include "crpropa/Source.h"
#include "crpropa/magneticField/MagneticField.h"

#include <stdint.h>

#include <string>

struct crp_run_stats;

namespace crpgpu {

/// B = b0 (-y, x, 0) / r with r = sqrt(x^2 + y^2): the analytic toroidal
/// field of the diffusion workload.  No reference class has this form
/// (ToroidalHaloField, GalacticMagneticField.h:17, has another).  getField
/// on the CPU; the plugin maps it to CRP_FIELD_TOROIDAL.
class ToroidalMagneticField : public crpropa::MagneticField {
    double b0;

public:
    explicit ToroidalMagneticField(double b0);
    crpropa::Vector3d getField(const crpropa::Vector3d &position) const;
    double getB0() const;
};

/// MaximumTrajectoryLength (BreakCondition.cpp:42) with the limit read per
/// candidate from the double property `key`.  No reference counterpart (the
/// reference's condition holds one limit).
class CandidateMaximumTrajectoryLength : public crpropa::AbstractCondition {
    std::string key;

public:
    explicit CandidateMaximumTrajectoryLength(const std::string &key = "MaximumTrajectoryLength");
    void process(crpropa::Candidate *candidate) const;
    std::string getPropertyKey() const;
    std::string getDescription() const;
};

class GpuModuleList : public crpropa::ModuleList {
public:
    enum Precision { FP64 = 0, MIXED = 1 };  // crp_precision

    GpuModuleList();
    ~GpuModuleList();

    /// ModuleList::run, same signatures (ModuleList.h:41-44).
    void run(crpropa::Candidate *candidate, bool recursive = true, bool secondariesFirst = false);
    void run(crpropa::ref_ptr<crpropa::Candidate> candidate, bool recursive = true,
             bool secondariesFirst = false);
    void run(const candidate_vector_t *candidates, bool recursive = true,
             bool secondariesFirst = false);
    void run(crpropa::SourceInterface *source, size_t count, bool recursive = true,
             bool secondariesFirst = false);

    /// FP64 (the reference's arithmetic) or MIXED (FP32 field and stage
    /// arithmetic, FP64 accumulation).  Default FP64.
    void setPrecision(Precision p);
    Precision getPrecision() const;
    /// Key of DiffusionSDE's counter-based random stream.  Default 0.
    void setSeed(uint64_t seed);
    /// Candidates per device batch in run(source, count) and
    /// run(candidates).  Default 2^20.
    void setBatchSize(size_t n);
    /// Run unsupported chains with ModuleList::run instead of throwing.
    void setCpuFallback(bool allow);

    /// Whether the chain maps onto the device path; *reason names the first
    /// module or field that does not.
    bool isSupported(std::string *reason = 0) const;
    /// The translated plan as text (fields, modules, parameters), for
    /// inspection; throws where isSupported() is false.
    std::string describePlan() const;
    /// Statistics of the last device run (steps, tries, launches, device ms).
    const crp_run_stats &getLastRunStats() const;
    /// Events (detections, rejections) replayed by the last run.
    uint64_t getLastRunEvents() const;

    std::string getDescription() const;

private:
    struct Impl;
    Impl *impl;
    GpuModuleList(const GpuModuleList &);
    GpuModuleList &operator=(const GpuModuleList &);
    void runDevice(const candidate_vector_t &candidates);
    void addStats(crp_run_stats &total, uint64_t &events) const;
};

}  // namespace crpgpu

#endif
