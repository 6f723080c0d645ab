// input.prm reader of the LBFlow command line.
//
// The file format is LBFlow's (solver/src/file/fileprm.cpp:297-456,
// 563-670): each line starts with a key token; the rest of the line is the
// value.  Keys starting with a digit define geometry labels as four quoted
// fields "TYPE" "value" "dir" "phase".  Values are read with the same stream
// conversions (numbers with operator>>, strings between the first pair of
// double quotes), so the same files parse to the same parameters and the same
// malformed files fail.  Validation messages follow
// FilePrm::ValidateSimulation (fileprm.cpp:136-295).
#ifndef LBF_HOST_PRM_H
#define LBF_HOST_PRM_H

#include <cstddef>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

namespace lbfhost {

enum LabelType { VD = 0x1, GV = 0x2, PB = 0x4, VB = 0x8, AB = 0x10, BB = 0x20, HF = 0x40, SD = 0x80 };

struct Label {
    LabelType type = VD;
    double value = 0.0;
    std::size_t dir = 0;
    std::size_t phase = 0;
};

class Params {
public:
    explicit Params(const std::string& path);

    // Required values: throw "the value may not be defined in parameter file."
    const std::string& gridFile() const { return req(gridFile_); }
    const std::vector<std::size_t>& dimension() const { return dimension_; }
    std::size_t directions() const { return req(directions_); }
    const std::string& fileType() const { return req(fileType_); }
    double latticeLen() const { return req(latticeLen_); }
    std::size_t tStart() const { return req(tStart_); }
    std::size_t tEnd() const { return req(tEnd_); }
    std::size_t tWrite() const { return req(tWrite_); }
    std::size_t tReport() const { return req(tReport_); }
    std::size_t tRestart() const { return req(tRestart_); }
    double stopError() const { return req(stopError_); }
    const std::string& outPath() const { return req(outPath_); }
    std::size_t reportDir() const { return req(reportDir_); }
    const std::vector<std::size_t>& reportSlice() const { return reportSlice_; }
    const std::string& fluidModel() const { return req(fluidModel_); }
    const std::string& equilModel() const { return req(equilModel_); }
    const std::vector<double>& relaxationTime() const { return relaxationTime_; }
    double latticeSpeed() const { return req(latticeSpeed_); }
    double alpha0() const { return req(alpha0_); }
    const std::vector<double>& density() const { return density_; }
    double surfaceTension() const { return req(surfaceTension_); }
    double interfaceThickness() const { return req(interfaceThickness_); }

    // Optional selectors with the reference's defaults.
    std::string selector(const std::string& key, const std::string& fallback,
                         const std::string& what) const;
    double wallSlipLength() const;

    // Label table; label() throws std::out_of_range for an undefined label.
    const Label& label(std::size_t value) const;
    bool hasLabel(std::size_t value) const { return labels_.count(value) != 0; }
    const std::map<std::size_t, Label>& labels() const { return labels_; }
    std::set<std::size_t> labelsOf(unsigned typeMask) const;

    void validate() const;   // FilePrm::ValidateSimulation
    std::size_t dims() const { return dimension_.size(); }

private:
    template <class T> static const T& req(const std::unique_ptr<T>& p)
    {
        if (!p) throw std::runtime_error("the value may not be defined in parameter file.");
        return *p;
    }
    std::map<std::string, std::string> raw_;
    std::unique_ptr<std::string> gridFile_, fileType_, outPath_, logPath_, fluidModel_, equilModel_;
    std::unique_ptr<std::size_t> directions_, tStart_, tEnd_, tWrite_, tReport_, tRestart_, reportDir_;
    std::unique_ptr<double> latticeLen_, stopError_, latticeSpeed_, alpha0_, contactAngle_,
        surfaceTension_, interfaceThickness_;
    std::vector<std::size_t> dimension_, reportSlice_;
    std::vector<double> relaxationTime_, density_;
    std::vector<std::string> phase_, components_;
    std::map<std::size_t, Label> labels_;
};

}  // namespace lbfhost

#endif
