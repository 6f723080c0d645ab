// The LBFlow run loop on the B200 engine.
#ifndef LBF_HOST_SIMULATION_H
#define LBF_HOST_SIMULATION_H

#include <chrono>
#include <cstdint>
#include <exception>
#include <ostream>
#include <string>
#include <thread>
#include <vector>

#include "lbflow.h"
#include "prm.h"

namespace lbfhost {

// "Time elapsed" logger with LBFlow's format (solver/src/helper/logger.cpp:25-75).
class StepLog {
public:
    explicit StepLog(std::ostream& os) : os_(os), t0_(now()) {}
    void log(const std::string& s, bool timer = true);
    void reset(bool autoReset = false) { auto_ = autoReset; t0_ = now(); }
    static double now();
    static std::string elapsed(double seconds);
private:
    std::ostream& os_;
    double t0_;
    bool auto_ = false;
};

// One file write in the background at a time, from a page-locked buffer the
// device fills (lbf_fields_dense_async / lbf_populations_dense_async), so the
// steps that follow an output run while the file is written.
class BackgroundWriter {
public:
    ~BackgroundWriter();
    // Joins the previous write and rethrows its failure.
    void wait();
    // A buffer of at least `count` doubles (kept across writes).
    double* buffer(std::size_t count);
    template <class F> void start(F&& write)
    {
        thread_ = std::thread([this, write]() {
            try { write(); } catch (...) { error_ = std::current_exception(); }
        });
    }
private:
    std::thread thread_;
    std::exception_ptr error_;
    double* buf_ = nullptr;
    std::size_t cap_ = 0;
};

class Simulation {
public:
    explicit Simulation(const Params& p);
    ~Simulation();
    Simulation(const Simulation&) = delete;
    Simulation& operator=(const Simulation&) = delete;
    void run(std::ostream& log);

private:
    void check(int rc, const char* what) const;
    void checkDevice() const;          // device error word -> the reference's exception
    void saveFields(std::size_t t);
    void saveCheckpoint(std::size_t t);
    void loadCheckpoint(std::size_t t);
    bool report(std::ostream& os);
    bool updateConvergence(std::ostream& os, bool scalarsStable, const double sums[6]);
    void writeTiming(std::ostream& os, double run) const;

    const Params& p_;
    bool color_;
    std::size_t D_, Q_, N_, phases_;
    std::vector<std::size_t> sz_;      // reference order sizes
    std::vector<uint8_t> geometry_;
    lbf_engine* e_ = nullptr;
    BackgroundWriter fieldWriter_, checkpointWriter_;
    double fluidNodes_ = 0;
    double seconds_[4] = {0, 0, 0, 0}; // INIT, NUMERICAL, FIELD, CHECKPOINT
    std::size_t completed_ = 0;
    // report state (the reference keeps these in function statics)
    bool hasReport_ = false;
    std::size_t stable_ = 0;
    double kOld_ = 0, sOld_[2] = {0, 0};
    std::size_t axis_ = 0, lo_ = 0, hi_ = 0;
    double cntLo_ = 0, cntHi_ = 0, kPar_ = 0;
};

}  // namespace lbfhost

#endif
