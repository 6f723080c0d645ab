// The LBFlow run loop on the B200 engine.
//
// Stage order, log lines, report arithmetic and convergence logic follow
// SCSP::Run / ColorFluid::Run (solver/src/lbm/scsp.cpp:46-114,
// colorfluid.cpp:109-212), SCSP::report / ColorFluid::report (scsp.cpp:304-372,
// colorfluid.cpp:814-915) and Simulator::updateConvergence
// (simulator.cpp:248-325).  The numerical work runs on the GPU in batches of
// steps between output events; the host synchronises only at those events.
#include "simulation.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <iomanip>
#include <limits>
#include <sstream>
#include <stdexcept>

#include "io.h"

namespace lbfhost {

namespace {
enum { INIT_T = 0, NUMERICAL_T = 1, FIELD_T = 2, CHECKPOINT_T = 3 };
// Qaxis of the reference lattices: the grid axis (reference order) of each
// axial direction (gridspace.cpp:95, 142).
std::size_t qaxis(std::size_t D, std::size_t dir)
{
    static const std::size_t a2[5] = {0, 1, 0, 1, 0};
    static const std::size_t a3[7] = {0, 2, 2, 1, 1, 0, 0};
    return D == 2 ? a2[dir] : a3[dir];
}
}  // namespace

double StepLog::now()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

std::string StepLog::elapsed(double time)
{
    const std::size_t it = static_cast<std::size_t>(time);
    const std::size_t days = it / 86400, hh = (it % 86400) / 3600, mm = (it % 3600) / 60, ss = it % 60;
    const double left = time - static_cast<double>(it) + ss;
    std::ostringstream os;
    os.precision(6);
    os << days << "d," << std::setw(2) << std::setfill('0') << hh << ":" << std::setw(2) << std::setfill('0')
       << mm << ":" << std::setw(9) << std::setfill('0') << std::setiosflags(std::ios::fixed) << left;
    return os.str();
}

void StepLog::log(const std::string& s, bool timer)
{
    os_ << s;
    if (timer) os_ << "Time elapsed: " << elapsed(now() - t0_) << std::endl;
    if (auto_) t0_ = now();
    os_.flush();
}

void Simulation::check(int rc, const char* what) const
{
    if (rc != LBF_OK) throw std::runtime_error(std::string(what) + ": " + lbf_last_error(e_));
}

void Simulation::checkDevice() const
{
    uint32_t bits = 0;
    check(lbf_status(e_, &bits), "lbf_status");
    if (bits & LBF_ERR_DENSITY)
        throw std::runtime_error(color_ ? "Non-finite or non-positive total fluid density."
                                        : "Non-finite or non-positive fluid density.");
    if (bits & LBF_ERR_COMPONENT) throw std::runtime_error("Negative component density outside roundoff tolerance.");
    if (bits & LBF_ERR_TAU) throw std::runtime_error("Invalid local relaxation time.");
    if (bits & LBF_ERR_VELOCITY) throw std::runtime_error("Non-finite fluid velocity.");
}

Simulation::Simulation(const Params& p) : p_(p)
{
    p.validate();
    color_ = p.fluidModel() == "color";
    D_ = p.dims();
    Q_ = p.directions();
    phases_ = color_ ? 2 : 1;
    sz_ = p.dimension();
    N_ = 1;
    for (std::size_t n : sz_) N_ *= n;
    geometry_ = loadGeometry(p.gridFile(), N_);
    bool used[256] = {};
    for (uint8_t v : geometry_) {
        if (!used[v]) p.label(v);   // throws for an undefined label, as the reference does
        used[v] = true;
    }
    if (p.reportDir() != 0) {
        const std::size_t axis = qaxis(D_, p.reportDir());
        for (std::size_t value : p.reportSlice())
            if (value >= sz_[axis]) throw std::invalid_argument("Report slice is outside the selected axis.");
    }
    if (!color_ && p.equilModel() != "SRT" && p.equilModel() != "MRT")
        throw std::invalid_argument("Invalid equilibrium model.");
    // fluid_nodes of the timing line (simulator.cpp:47-56).
    for (uint8_t v : geometry_) {
        const LabelType t = p.label(v).type;
        fluidNodes_ += (t == VD || t == GV || t == VB || t == PB || (color_ && t == HF)) ? 1.0 : 0.0;
    }

    lbf_config c{};
    c.dims = (uint32_t)D_;
    c.nx = (uint32_t)sz_[D_ - 1];
    c.ny = (uint32_t)sz_[D_ - 2];
    c.nz = D_ == 3 ? (uint32_t)sz_[0] : 1;
    c.model = color_ ? LBF_MODEL_COLOR : LBF_MODEL_SCSP;
    c.collision = p.equilModel() == "MRT" ? LBF_MRT : LBF_SRT;
    // Optional extension key (ignored by the reference's parser): population storage.
    const std::string storage = p.selector("populationStorage", "fp64", "populationStorage");
    c.storage = storage == "fp16" ? LBF_STORE_FP16 : storage == "bf16" ? LBF_STORE_BF16
              : storage == "fp32" ? LBF_STORE_FP32 : storage == "bfp16" ? LBF_STORE_BFP16 : LBF_STORE_FP64;
    if (storage != "fp64" && storage != "fp32" && storage != "fp16" && storage != "bf16" && storage != "bfp16")
        throw std::invalid_argument("populationStorage must be fp64, fp32, fp16, bf16 or bfp16.");
    const char* dev = std::getenv("LBFLOW_DEVICE");
    c.device = dev ? std::atoi(dev) : 0;
    for (std::size_t k = 0; k < 2; ++k) {
        c.tau[k] = p.relaxationTime()[std::min(k, phases_ - 1)];
        c.rho[k] = p.density()[std::min(k, phases_ - 1)];
    }
    c.alpha0 = p.alpha0();
    c.sigma = color_ ? p.surfaceTension() : 0.0;
    c.beta = color_ ? p.interfaceThickness() : 0.0;
    std::vector<lbf_label> labels(256);
    for (const auto& kv : p.labels()) {
        if (kv.first > 255) continue;
        lbf_label& l = labels[kv.first];
        l.type = kv.second.type;
        l.dir = (int32_t)kv.second.dir;
        l.phase = (int32_t)kv.second.phase;
        l.value = kv.second.value;
    }
    const int rc = lbf_create(&c, labels.data(), geometry_.data(), &e_);
    if (rc != LBF_OK) throw std::runtime_error(std::string("engine: ") + lbf_last_error(nullptr));
    // Optional extension key: checkpoints with the reference's values at
    // solid voxels too (lbf_keep_solid_populations).
    const std::string solids = p.selector("solidPopulations", "zero", "solidPopulations");
    if (solids != "zero" && solids != "stream")
        throw std::invalid_argument("solidPopulations must be zero or stream.");
    if (solids == "stream" && lbf_keep_solid_populations(e_) != LBF_OK)
        throw std::runtime_error(std::string("engine: ") + lbf_last_error(e_));

    if (p.reportDir() != 0) {
        axis_ = qaxis(D_, p.reportDir());
        const auto& sl = p.reportSlice();
        lo_ = *std::min_element(sl.begin(), sl.end());
        hi_ = *std::max_element(sl.begin(), sl.end());
        // Simulator::getKPar (simulator.cpp:151-160).
        const double viscosity = (p.relaxationTime()[0] - 0.5) * p.latticeSpeed() / 3;
        const double len = static_cast<double>(sl.back() - sl.front());
        double area = 1;
        for (std::size_t d = 0; d < D_; ++d)
            if (d != axis_) area *= sz_[d];
        kPar_ = len * viscosity / area * std::pow(p.latticeLen(), 2) * 1.0e12;
    }
}

BackgroundWriter::~BackgroundWriter()
{
    if (thread_.joinable()) thread_.join();
    lbf_host_free(buf_);
}

void BackgroundWriter::wait()
{
    if (thread_.joinable()) thread_.join();
    if (error_) {
        std::exception_ptr e = error_;
        error_ = nullptr;
        std::rethrow_exception(e);
    }
}

double* BackgroundWriter::buffer(std::size_t count)
{
    if (count > cap_) {
        lbf_host_free(buf_);
        buf_ = nullptr;
        cap_ = 0;
        void* p = nullptr;
        if (lbf_host_alloc(count * sizeof(double), &p) != LBF_OK)
            throw std::runtime_error(std::string("output buffer: ") + lbf_last_error(nullptr));
        buf_ = static_cast<double*>(p);
        cap_ = count;
    }
    return buf_;
}

Simulation::~Simulation()
{
    // Finish the files in flight (their failures no longer matter here), then
    // release the engine.
    try { fieldWriter_.wait(); } catch (...) {}
    try { checkpointWriter_.wait(); } catch (...) {}
    if (e_) lbf_destroy(e_);
}

// Output::Save (filevti.cpp:39-172): the device writes the dense arrays into a
// page-locked buffer; the file is written in the background.
void Simulation::saveFields(std::size_t t)
{
    fieldWriter_.wait();
    const std::size_t n = (1 + (color_ ? 1 : 0) + D_) * N_;
    double* buf = fieldWriter_.buffer(n);
    check(lbf_fields_dense_async(e_, buf, n), "lbf_fields_dense_async");
    check(lbf_synchronize(e_), "lbf_synchronize");
    const std::vector<std::string> scalars = color_ ? std::vector<std::string>{"r0", "r1"}
                                                    : std::vector<std::string>{"density"};
    const std::string path = stepName(p_.outPath(), t, ".vti");
    const std::vector<std::size_t> sz = sz_;
    const std::string vec = color_ ? "v" : "velocity";
    const int comps = (int)D_;
    fieldWriter_.start([path, sz, scalars, vec, comps, buf]() { writeVtiBlocks(path, sz, scalars, vec, comps, buf); });
}

// saveRst (scsp.cpp:277-302; colorfluid.cpp:766-812) with the finite check of
// validatePopulations (simulator.cpp:327-333) done by the device; the sidecar
// follows the population file in the background write.
void Simulation::saveCheckpoint(std::size_t t)
{
    checkDevice();
    checkpointWriter_.wait();
    const std::size_t count = phases_ * Q_ * N_;
    double* buf = checkpointWriter_.buffer(count);
    check(lbf_populations_dense_async(e_, buf, count), "lbf_populations_dense_async");
    uint32_t bits = 0;
    check(lbf_status(e_, &bits), "lbf_status");
    if (bits & LBF_ERR_OUTPUT)
        throw std::runtime_error("Non-finite post-collision population; no restart will be written.");
    const std::string name = stepName(p_.outPath(), t, ".rst");
    const std::size_t phases = phases_, D = D_, Q = Q_;
    const std::vector<std::size_t> sz = sz_;
    checkpointWriter_.start([name, buf, count, t, phases, D, Q, sz]() {
        writeCheckpoint(name, buf, count);
        writeCheckpointMeta(name, t, phases, D, Q, sz);
    });
}

void Simulation::loadCheckpoint(std::size_t t)
{
    const std::string name = stepName(p_.outPath(), t, ".rst");
    validateCheckpoint(name, t, phases_, D_, Q_, sz_);
    const std::size_t count = phases_ * Q_ * N_;
    std::vector<double> f = readCheckpoint(name, count);
    check(lbf_set_populations(e_, f.data(), count), "lbf_set_populations");
    hasReport_ = false;
    stable_ = 0;
}

bool Simulation::updateConvergence(std::ostream& os, bool scalarsStable, const double s[6])
{
    const double tol = p_.stopError();
    const double count = static_cast<double>(D_) * static_cast<double>(N_);
    if (!std::isfinite(s[0]) || !std::isfinite(s[1]) || !std::isfinite(s[2]) || count <= 0.0)
        throw std::runtime_error("Invalid global velocity residual.");
    const double rmsChange = std::sqrt(s[0] / count);
    const double residual = s[1] > 0.0 ? std::sqrt(s[0] / s[1]) : 0.0;
    const bool velocityStable = rmsChange <= 1e-12 || residual < tol;
    const double adjacentRms = std::sqrt(s[2] / count);
    const double adjacentResidual = s[1] > 0.0 ? std::sqrt(s[2] / s[1]) : 0.0;
    const bool adjacentStable = adjacentRms <= 1e-12 || adjacentResidual < tol;
    const double pc0 = color_ ? s[3] : 0.0, pc1 = color_ ? s[4] : 0.0;
    stable_ = scalarsStable && velocityStable && adjacentStable && std::max(pc0, pc1) < tol ? stable_ + 1 : 0;
    os << " - velocityResidual = " << residual << ", velocityRmsChange = " << rmsChange
       << ", adjacentVelocityResidual = " << adjacentResidual << ", adjacentVelocityRmsChange = " << adjacentRms
       << ", maxPhaseChange = " << pc0 << ", adjacentMaxPhaseChange = " << pc1
       << ", stableReports = " << stable_ << "/3" << std::endl;
    return stable_ >= 3;
}

bool Simulation::report(std::ostream& os)
{
    if (p_.reportDir() == 0) return false;
    try {
        const uint32_t ours = (uint32_t)(D_ - 1 - axis_);
        double r[10];
        check(lbf_report_sums(e_, ours, (uint32_t)lo_, (uint32_t)hi_, r), "lbf_report_sums");
        if (cntLo_ == 0 && cntHi_ == 0) { cntLo_ = r[7]; cntHi_ = r[8]; }
        const double maxErr = p_.stopError();
        const double Q = r[0] / double(hi_ - lo_ + 1);
        double dP;
        bool scalarsStable;
        if (!color_) {
            dP = (r[3] / cntLo_ - r[5] / cntHi_) / 3.0;
            if (!std::isfinite(dP) || !std::isfinite(Q)) throw std::runtime_error("Non-finite single-phase report state.");
        } else {
            const double a0 = p_.alpha0();
            const double a1 = 1 - p_.density()[0] / p_.density()[1] * (1 - a0);
            const double pf = Q_ == 9 ? 3.0 / 5.0 : 1.0 / 2.0;
            const double r2p[2] = {(1.0 - a0) * pf, (1.0 - a1) * pf};
            const double stc0 = r[1] / p_.density()[0], stc1 = r[2] / p_.density()[1];
            const double stcT = stc0 + stc1;
            const double S[2] = {stc0 / stcT, stc1 / stcT};
            const double errS[2] = {std::abs(S[0] - sOld_[0]), std::abs(S[1] - sOld_[1])};
            sOld_[0] = S[0]; sOld_[1] = S[1];
            dP = (r[3] * r2p[0] + r[4] * r2p[1]) / cntLo_ - (r[5] * r2p[0] + r[6] * r2p[1]) / cntHi_;
            if (!std::isfinite(S[0]) || !std::isfinite(S[1]) || !std::isfinite(errS[0]) ||
                !std::isfinite(errS[1]) || !std::isfinite(dP) || !std::isfinite(Q))
                throw std::runtime_error("Non-finite two-phase report state.");
            os << std::setprecision(6) << std::fixed << " - S0 = " << S[0] * 100 << "%, " << "dS0 = "
               << errS[0] * 100 << "%" << std::endl << " - S1 = " << S[1] * 100 << "%, " << "dS1 = "
               << errS[1] * 100 << "%" << std::endl;
            scalarsStable = std::max(errS[0], errS[1]) < maxErr;
        }
        const bool hasDrop = std::abs(dP) > 1e-14;
        const double K = hasDrop ? kPar_ * Q / dP : 0.0;
        const double errK = hasDrop ? std::abs(K - kOld_) / std::max(std::abs(K), 1e-30) : 0.0;
        if (!std::isfinite(K) || !std::isfinite(errK)) throw std::runtime_error("Non-finite apparent permeability.");
        kOld_ = K;
        os << std::setprecision(6) << std::scientific << " - dP = " << dP << "(mu/lu/ts^2), " << "Q = " << Q
           << "(lu^3/ts)" << std::endl << " - K = " << K << "(um^2), " << std::fixed << "errK = "
           << errK * 100.0 << "%" << std::endl;
        if (!hasDrop) os << " - pressure-based permeability unavailable: zero pressure drop" << std::endl;
        if (!color_) scalarsStable = !hasDrop || errK < maxErr;
        else scalarsStable = scalarsStable && (!hasDrop || errK < maxErr);
        double s[6] = {0, 0, 0, 0, 0, 0};
        if (!hasReport_) {
            check(lbf_convergence(e_, 1, s), "lbf_convergence");
            hasReport_ = true;
            stable_ = 0;
            return false;
        }
        check(lbf_convergence(e_, 0, s), "lbf_convergence");
        return updateConvergence(os, scalarsStable, s);
    } catch (std::exception& e) {
        os << e.what();
        throw;
    }
}

void Simulation::writeTiming(std::ostream& os, double run) const
{
    std::ostringstream s;
    s << std::setprecision(17) << "LBFlowTiming {\"schema\":1,\"ranks\":1"
      << ",\"completed_steps\":" << completed_ << ",\"fluid_nodes\":" << fluidNodes_
      << ",\"total_voxels\":" << N_ << ",\"initialization_seconds_max\":" << seconds_[INIT_T]
      << ",\"numerical_seconds_max\":" << seconds_[NUMERICAL_T]
      << ",\"fields_diagnostics_seconds_max\":" << seconds_[FIELD_T]
      << ",\"checkpoint_seconds_max\":" << seconds_[CHECKPOINT_T] << ",\"run_seconds_max\":" << run << "}\n";
    os << s.str();
}

void Simulation::run(std::ostream& log)
{
    const double runStart = StepLog::now();
    StepLog procLog(log);
    procLog.reset(true);
    procLog.log("Initializing...", false);
    const std::size_t t0 = p_.tStart(), tEnd = p_.tEnd();
    if (t0 != 0) {
        const double b = StepLog::now();
        loadCheckpoint(t0);
        seconds_[CHECKPOINT_T] += StepLog::now() - b;
    } else {
        double b = StepLog::now();
        check(lbf_initialize(e_), "lbf_initialize");
        check(lbf_synchronize(e_), "lbf_synchronize");
        checkDevice();
        seconds_[INIT_T] += StepLog::now() - b;
        b = StepLog::now();
        saveFields(t0);
        seconds_[FIELD_T] += StepLog::now() - b;
    }
    procLog.log("Done!\t");

    const std::size_t tw = p_.tWrite(), tr = p_.tReport(), ts = p_.tRestart();
    const bool reporting = p_.reportDir() != 0;
    auto needsAdjacent = [&](std::size_t t) { return reporting && t <= tEnd && (t % tw == 0 || t % tr == 0); };
    std::size_t t = t0;
    while (t < tEnd) {
        std::size_t te = tEnd;
        te = std::min(te, (t / tw + 1) * tw);
        te = std::min(te, (t / tr + 1) * tr);
        te = std::min(te, (t / ts + 1) * ts);
        const bool isWrite = te % tw == 0, isReport = te % tr == 0, isRestart = te % ts == 0;
        const std::size_t n = te - t;
        const uint32_t last = ((isWrite || isReport) ? LBF_STEP_MACROS : 0) |
                              (needsAdjacent(te + 1) ? LBF_STEP_ADJACENT : 0);
        double b = StepLog::now();
        if (n >= 2) check(lbf_step(e_, (uint32_t)(n - 1), needsAdjacent(te) ? LBF_STEP_ADJACENT : 0), "lbf_step");
        check(lbf_step(e_, 1, last), "lbf_step");
        check(lbf_synchronize(e_), "lbf_synchronize");
        seconds_[NUMERICAL_T] += StepLog::now() - b;
        checkDevice();
        t = te;
        bool converged = false;
        b = StepLog::now();
        if (isWrite) {
            std::ostringstream ss;
            ss << "Step " << t << " - ";
            procLog.log(ss.str());
            saveFields(t);
            converged = report(log);
        } else if (isReport) {
            std::ostringstream ss;
            ss << "Step " << t << " - ";
            procLog.log(ss.str());
            converged = report(log);
        }
        seconds_[FIELD_T] += StepLog::now() - b;
        if (converged || isRestart) {
            b = StepLog::now();
            saveCheckpoint(t);
            seconds_[CHECKPOINT_T] += StepLog::now() - b;
        }
        completed_ += n;
        if (converged) break;
    }
    // The files still being written belong to their output categories.
    double b = StepLog::now();
    fieldWriter_.wait();
    seconds_[FIELD_T] += StepLog::now() - b;
    b = StepLog::now();
    checkpointWriter_.wait();
    seconds_[CHECKPOINT_T] += StepLog::now() - b;
    writeTiming(log, StepLog::now() - runStart);
}

}  // namespace lbfhost
