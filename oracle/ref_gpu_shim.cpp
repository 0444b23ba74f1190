/*
 * ref_gpu_shim.cpp -- TEST INFRASTRUCTURE, not product code.
 *
 * Builds the reference's own chain objects from a crp_plan_desc (the same
 * builder as ref_shim.cpp) into the plugin's crpgpu::GpuModuleList and runs
 * them through it, so that the tests can compare the plugin's device run of
 * an unmodified CRPropa chain with the reference's ModuleList::run on the
 * same Candidate objects.  Loaded only by tests/.
 */
#include "ref_chain.h"

#include "GpuModuleList.h"

#include "crpropa/ParticleID.h"
#include "crpropa/Random.h"
#include "crpropa/Source.h"
#include "crpropa/Units.h"
#include "crpropa/module/BreakCondition.h"
#include "crpropa/module/Observer.h"
#include "crpropa/module/RestrictToRegion.h"
#include "crpropa/module/SimplePropagation.h"
#include "crpropa/module/TextOutput.h"

#include <omp.h>
#include <signal.h>
#include <unistd.h>

#include <algorithm>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>

using namespace crpropa;
using namespace crp_ref;

namespace {

std::string g_error;

struct PluginHelpers : Helpers {
    MagneticField *toroidal(double b0) const { return new crpgpu::ToroidalMagneticField(b0); }
    AbstractCondition *perCandidateLength() const {
        return new crpgpu::CandidateMaximumTrajectoryLength("CrpMaxLength");
    }
};

void copy_text(const std::string &s, char *buf, size_t size) {
    if (!buf || !size) return;
    size_t n = std::min(s.size(), size - 1);
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
}

// A detection action that sends SIGINT to the process at its first event:
// an interruption at a known point of a run.
struct SignalAtFirstDetection : public Module {
    mutable bool fired = false;
    void process(Candidate *) const {
        if (!fired) {
            fired = true;
            kill(getpid(), SIGINT);
        }
    }
};

volatile sig_atomic_t g_reraised = 0;
extern "C" void shim_on_signal(int sig) { g_reraised = sig; }

crpgpu::GpuModuleList *make_list(int precision, uint64_t seed) {
    crpgpu::GpuModuleList *g = new crpgpu::GpuModuleList();
    g->setPrecision(precision == 1 ? crpgpu::GpuModuleList::MIXED : crpgpu::GpuModuleList::FP64);
    g->setSeed(seed);
    return g;
}

}  // namespace

extern "C" {

const char *ref_gpu_last_error() { return g_error.c_str(); }

/* Run the chain of `desc` through GpuModuleList::run(candidate_vector_t*)
 * on the candidates (in/out), with record actions as in ref_run. */
int ref_gpu_run(const crp_plan_desc *desc, const crp_candidates *c, uint64_t n, crp_records *rec,
                int precision, uint64_t seed, crp_run_stats *stats, uint64_t *events) {
    try {
        ensure_data_path();
        PluginHelpers h;
        Built b;
        crpgpu::GpuModuleList *g = make_list(precision, seed);
        build_chain(desc, rec, b, &h, g, false, 0, 0);
        ModuleList::candidate_vector_t cands;
        load_candidates(c, n, cands);
        g->run(&cands);
        store_candidates(cands, c);
        if (stats) *stats = g->getLastRunStats();
        if (events) *events = g->getLastRunEvents();
        return 0;
    } catch (std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

/* The same with TextOutput(path, output_type) as every observer's action. */
int ref_gpu_run_textout(const crp_plan_desc *desc, const crp_candidates *c, uint64_t n,
                        const char *path, int output_type, int precision, uint64_t seed,
                        uint64_t serial0) {
    try {
        ensure_data_path();
        PluginHelpers h;
        Built b;
        {
            crpgpu::GpuModuleList *g = make_list(precision, seed);
            build_chain(desc, 0, b, &h, g, false, path, output_type);
            Candidate::setNextSerialNumber(serial0);
            ModuleList::candidate_vector_t cands;
            load_candidates(c, n, cands);
            g->run(&cands);
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

/* Source of the reference (Source.cpp): SourcePosition(pos),
 * SourceParticleType(id), SourcePowerLawSpectrum(emin, emax, index),
 * SourceIsotropicEmission, run through `count` candidates with
 * run(source, count): on the plugin when gpu != 0 (batches of `batch`),
 * else on the reference's ModuleList with one thread.  Random::seedThreads
 * (seed) first; serial numbers from serial0.  The chain's observers write
 * TextOutput(path, output_type). */
int ref_run_source_textout(const crp_plan_desc *desc, int gpu, int precision, const double *pos,
                           int32_t id, double emin, double emax, double index, uint64_t count,
                           uint64_t batch, const char *path, int output_type, uint32_t seed,
                           uint64_t serial0, crp_run_stats *stats) {
    try {
        ensure_data_path();
        PluginHelpers h;
        Built b;
        {
            ref_ptr<Source> src = new Source();
            src->add(new SourcePosition(Vector3d(pos[0], pos[1], pos[2])));
            src->add(new SourceParticleType(id));
            src->add(new SourcePowerLawSpectrum(emin, emax, index));
            src->add(new SourceIsotropicEmission());
            crpgpu::GpuModuleList *g = 0;
            if (gpu) {
                g = make_list(precision, 0);
                if (batch) g->setBatchSize(batch);
            }
            build_chain(desc, 0, b, gpu ? &h : 0, g, false, path, output_type);
            Candidate::setNextSerialNumber(serial0);
            Random::seedThreads(seed);
            omp_set_num_threads(1);
            std::streambuf *old = std::cout.rdbuf();
            std::ostringstream sink;
            std::cout.rdbuf(sink.rdbuf());
            if (g)
                g->run(src.get(), count);
            else
                b.sim->run(src.get(), count);
            std::cout.rdbuf(old);
            if (g && stats) *stats = g->getLastRunStats();
        }
        b.sim = 0;
        return 0;
    } catch (std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

/* ModuleList::run(candidate_vector_t*) interrupted by SIGINT: every
 * Observer of the chain gets SignalAtFirstDetection as its detection action
 * and the run a TextOutput(path) as its interrupt action
 * (ModuleList::setInterruptAction).  On the plugin when gpu != 0 (batches of
 * `batch`), else on the reference's ModuleList with one thread.  The
 * harness catches the signal the run raises again at its end and reports it
 * in *reraised; the caller's SIGINT handler is restored afterwards. */
int ref_run_interrupted(const crp_plan_desc *desc, const crp_candidates *c, uint64_t n, int gpu,
                        uint64_t batch, const char *path, int *reraised) {
    struct sigaction sa, old;
    std::memset(&sa, 0, sizeof(sa));
    sa.sa_handler = shim_on_signal;
    sigaction(SIGINT, &sa, &old);
    g_reraised = 0;
    int rc = 0;
    try {
        ensure_data_path();
        PluginHelpers h;
        Built b;
        {
            crpgpu::GpuModuleList *g = 0;
            if (gpu) {
                g = make_list(desc->precision, desc->seed);
                if (batch) g->setBatchSize(batch);
            }
            build_chain(desc, 0, b, gpu ? &h : 0, g, false, 0, 0);
            ref_ptr<Module> signal_action = new SignalAtFirstDetection();
            for (ModuleList::iterator it = b.sim->begin(); it != b.sim->end(); ++it) {
                Observer *obs = dynamic_cast<Observer *>(it->get());
                if (obs) obs->onDetection(signal_action.get());
            }
            ref_ptr<TextOutput> interrupt = new TextOutput(path);
            b.sim->setInterruptAction(interrupt.get());
            ModuleList::candidate_vector_t cands;
            load_candidates(c, n, cands);
            omp_set_num_threads(1);
            std::streambuf *old_out = std::cout.rdbuf();
            std::ostringstream sink;
            std::cout.rdbuf(sink.rdbuf());
            if (g)
                g->run(&cands);  // run() is not virtual: call the plugin's own
            else
                b.sim->run(&cands);
            std::cout.rdbuf(old_out);
            store_candidates(cands, c);
            interrupt->close();
        }
        b.sim = 0;
    } catch (std::exception &e) {
        g_error = e.what();
        rc = 1;
    }
    *reraised = g_reraised;
    sigaction(SIGINT, &old, 0);
    return rc;
}

/* The plugin's translation of the chain of `desc` (no device needed):
 * returns 1 and the plan text if the chain is on the device path, 0 and the
 * reason otherwise.  extra: 1 appends a SimplePropagation, 2 a
 * MinimumEnergy, 3 sets MaximumTrajectoryLength observer positions, 4
 * appends a RestrictToRegion, 5 sets setMakeRejectedInactive(false) on the
 * MaximumTrajectoryLength. */
int ref_gpu_describe(const crp_plan_desc *desc, int extra, char *buf, size_t size) {
    try {
        ensure_data_path();
        PluginHelpers h;
        Built b;
        crpgpu::GpuModuleList *g = make_list(desc->precision, desc->seed);
        build_chain(desc, 0, b, &h, g, false, 0, 0);
        if (extra == 1) g->add(new SimplePropagation());
        if (extra == 2) g->add(new MinimumEnergy(1 * EeV));
        for (ModuleList::iterator it = g->begin(); it != g->end(); ++it) {
            MaximumTrajectoryLength *m = dynamic_cast<MaximumTrajectoryLength *>(it->get());
            if (m && extra == 3) m->addObserverPosition(Vector3d(0.));
            if (m && extra == 5) m->setMakeRejectedInactive(false);
        }
        if (extra == 4)
            g->add(new RestrictToRegion(new MaximumTrajectoryLength(1 * Mpc), new Sphere(Vector3d(0.), 1 * Mpc)));
        std::string why;
        if (!g->isSupported(&why)) {
            copy_text(why, buf, size);
            return 0;
        }
        copy_text(g->describePlan(), buf, size);
        return 1;
    } catch (std::exception &e) {
        g_error = e.what();
        copy_text(std::string("error: ") + e.what(), buf, size);
        return -1;
    }
}

/* run() of an unsupported chain (SimplePropagation appended): 1 if it threw
 * with the reason, 0 if it ran. */
int ref_gpu_unsupported_throws(const crp_plan_desc *desc, char *buf, size_t size) {
    ensure_data_path();
    PluginHelpers h;
    Built b;
    crpgpu::GpuModuleList *g = make_list(desc->precision, desc->seed);
    build_chain(desc, 0, b, &h, g, false, 0, 0);
    g->add(new SimplePropagation());
    ModuleList::candidate_vector_t cands;
    cands.push_back(new Candidate(nucleusId(1, 1), 1 * EeV));
    try {
        g->run(&cands);
    } catch (std::exception &e) {
        copy_text(e.what(), buf, size);
        return 1;
    }
    return 0;
}

}  // extern "C"
