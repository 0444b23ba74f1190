/*
 * ref_chain.h -- TEST INFRASTRUCTURE, not product code.
 *
 * The chain builder of ref_shim.cpp, shared with ref_gpu_shim.cpp: it turns
 * a crp_plan_desc into the reference's own module objects (PropagationBP/CK,
 * DiffusionSDE, MagneticFieldGrid, ..., MaximumTrajectoryLength, Observer),
 * added to a given ModuleList (the reference's, or the GPU plugin's
 * GpuModuleList), and converts crp_candidates arrays to and from the
 * reference's Candidate objects.
 */
#ifndef CRP_REF_CHAIN_H
#define CRP_REF_CHAIN_H

#include "crp_gpu.h"

#include "crpropa/Candidate.h"
#include "crpropa/Module.h"
#include "crpropa/ModuleList.h"
#include "crpropa/magneticField/MagneticField.h"

#include <stdint.h>

#include <string>
#include <vector>

namespace crp_ref {

/* Counts process() calls of the chain, per OpenMP thread. */
class StepCounter : public crpropa::Module {
public:
    mutable std::vector<uint64_t> perThread;
    StepCounter();
    void process(crpropa::Candidate *c) const;
    uint64_t total() const;
};

/* Output type that asks build_chain for a ParticleCollector (clone on) as
 * the observers' detection action instead of a TextOutput; finish_outputs()
 * dumps the first one to the output path (ParticleCollector::dump,
 * ParticleCollector.cpp:62: TextOutput Everything). */
const int kCollectorOutput = 100;

struct Built {
    crpropa::ref_ptr<crpropa::ModuleList> sim;
    crpropa::ref_ptr<crpropa::MagneticField> field;
    std::vector<crpropa::ref_ptr<crpropa::Referenced> > keep;  // spectra, grids
    crpropa::ref_ptr<StepCounter> counter;
    std::vector<crpropa::ref_ptr<crpropa::Module> > collectors;
    std::string collector_path;
};

/* Dumps the chain's ParticleCollector, if any (call after the run). */
void finish_outputs(Built &b);

/* Factories for the two helpers without a reference class (toroidal field,
 * per-candidate maximum length); null: ref_shim.cpp's own. */
struct Helpers {
    virtual ~Helpers() {}
    virtual crpropa::MagneticField *toroidal(double b0) const = 0;
    virtual crpropa::AbstractCondition *perCandidateLength() const = 0;
};

void ensure_data_path();

/* Build the chain of `d` into `sim` (a new ModuleList if null).  Observers
 * get a TextOutput(text_output, text_type) detection action when text_output
 * is given, else a record action when the module asks for records.
 * count_steps appends a StepCounter. */
void build_chain(const crp_plan_desc *d, crp_records *rec, Built &b, const Helpers *h,
                 crpropa::ModuleList *sim, bool count_steps, const char *text_output,
                 int text_type);

/* Candidates from arrays: Candidate(id, E, pos, dir), previous position,
 * length, time, next step, active; properties CrpIndex (and CrpMaxLength). */
void load_candidates(const crp_candidates *c, uint64_t n,
                     crpropa::ModuleList::candidate_vector_t &cands);
void store_candidates(const crpropa::ModuleList::candidate_vector_t &cands,
                      const crp_candidates *c);

}  // namespace crp_ref

#endif
