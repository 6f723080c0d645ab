// input.prm reader (see prm.h).
#include "prm.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>

namespace lbfhost {

namespace {

// Value conversions with LBFlow's semantics (fileprm.cpp:491-561).
bool parseOne(const std::string& s, std::size_t* v) { std::istringstream is(s); is >> *v; return !is.fail(); }
bool parseOne(const std::string& s, double* v) { std::istringstream is(s); is >> *v; return !is.fail(); }
bool parseOne(const std::string& s, std::string* v)
{
    v->clear();
    std::istringstream is(s);
    char c;
    while (is.get(c) && c != '"') {}
    while (is.get(c) && c != '"') v->push_back(c);
    return !is.fail();
}
bool parseList(const std::string& s, std::vector<std::size_t>* v)
{
    v->clear();
    std::istringstream is(s);
    while (is) {
        int i;
        is >> i;
        if (is.fail()) break;
        v->push_back(static_cast<std::size_t>(i));
    }
    return !v->empty();
}
bool parseList(const std::string& s, std::vector<double>* v)
{
    v->clear();
    std::istringstream is(s);
    while (is) {
        double d;
        is >> d;
        if (is.fail()) break;
        v->push_back(d);
    }
    return !v->empty();
}
bool parseList(const std::string& s, std::vector<std::string>* v)
{
    v->clear();
    std::istringstream is(s);
    while (is) {
        std::string out;
        char c;
        while (is.get(c) && c != '"') {}
        while (is.get(c) && c != '"') out.push_back(c);
        if (is.fail()) break;
        v->push_back(out);
    }
    return !v->empty();
}

template <class T>
void set(const std::string& s, std::unique_ptr<T>* p)
{
    std::unique_ptr<T> v(new T());
    if (parseOne(s, v.get())) *p = std::move(v);
    else p->reset();
}

// Label field conversions (fileprm.cpp:605-631): an unparsable required field throws.
double fieldDouble(const std::string& s)
{
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str()) throw std::invalid_argument("IdxHead::str2d() - double value not defined");
    return v;
}
std::size_t fieldIndex(const std::string& s)
{
    char* end = nullptr;
    const unsigned long v = std::strtoul(s.c_str(), &end, 10);
    if (end == s.c_str()) throw std::invalid_argument("IdxHead::str2ul() - unsigned long value not defined");
    return v;
}

Label makeLabel(const std::vector<std::string>& f)
{
    if (f.size() < 4) throw std::invalid_argument("FilePrm::IDX::IDX() - insufficient val size.");
    Label l;
    const std::string& t = f[0];
    if (t == "VD") { l.type = VD; l.phase = fieldIndex(f[3]); }
    else if (t == "GV" || t == "PB" || t == "VB") {
        l.type = t == "GV" ? GV : (t == "PB" ? PB : VB);
        l.value = fieldDouble(f[1]);
        l.dir = fieldIndex(f[2]);
        l.phase = fieldIndex(f[3]);
    }
    else if (t == "AB") l.type = AB;
    else if (t == "BB") l.type = BB;
    else if (t == "SD") { l.type = SD; l.value = fieldDouble(f[1]); }
    else if (t == "HF") { l.type = HF; l.phase = fieldIndex(f[3]); }
    else throw std::invalid_argument("FilePrm::IDXVAL::IDXVAL() - unrecognized index descriptor type");
    return l;
}

}  // namespace

Params::Params(const std::string& path)
{
    {
        std::FILE* probe = std::fopen(path.c_str(), "r");
        if (!probe) throw std::runtime_error("FilePrm::Load() - Input file does not exist.");
        std::fclose(probe);
    }
    std::ifstream in(path);
    if (!in.is_open()) throw std::runtime_error("FilePrm::Load() - Failed to load input file");
    for (std::string key; in >> key;) {
        std::string rest;
        std::getline(in, rest);
        if (std::isalnum(static_cast<unsigned char>(key[0]))) raw_[key] = rest;
    }
    // Keys are processed in sorted order, as LBFlow's std::map does.
    for (const auto& kv : raw_) {
        const std::string& k = kv.first;
        const std::string& v = kv.second;
        if (k == "gridFile") set(v, &gridFile_);
        else if (k == "dimension") parseList(v, &dimension_);
        else if (k == "directions") set(v, &directions_);
        else if (k == "fileType") set(v, &fileType_);
        else if (k == "latticeLen") set(v, &latticeLen_);
        else if (k == "startTime") set(v, &tStart_);
        else if (k == "endTime") set(v, &tEnd_);
        else if (k == "writeInterval") set(v, &tWrite_);
        else if (k == "reportInterval") set(v, &tReport_);
        else if (k == "restartInterval") set(v, &tRestart_);
        else if (k == "stopError") set(v, &stopError_);
        else if (k == "outPath") set(v, &outPath_);
        else if (k == "logPath") set(v, &logPath_);
        else if (k == "reportDir") set(v, &reportDir_);
        else if (k == "reportSlice") parseList(v, &reportSlice_);
        else if (k == "fluidModel") set(v, &fluidModel_);
        else if (k == "equilModel") set(v, &equilModel_);
        else if (k == "rexlationTime") parseList(v, &relaxationTime_);
        else if (k == "latticeSpeed") set(v, &latticeSpeed_);
        else if (k == "alpha0") set(v, &alpha0_);
        else if (k == "density") parseList(v, &density_);
        else if (k == "phase") parseList(v, &phase_);
        else if (k == "contactAngle") set(v, &contactAngle_);
        else if (k == "surfaceTension") set(v, &surfaceTension_);
        else if (k == "interfaceThickness") set(v, &interfaceThickness_);
        else if (k == "components") parseList(v, &components_);
        else {
            char* end = nullptr;
            const unsigned long idx = std::strtoul(k.c_str(), &end, 10);
            if (end == k.c_str()) continue;   // not a label line (selectors are read on demand)
            std::vector<std::string> fields;
            if (parseList(v, &fields)) labels_[idx] = makeLabel(fields);
        }
    }
}

std::string Params::selector(const std::string& key, const std::string& fallback,
                             const std::string& what) const
{
    const auto it = raw_.find(key);
    if (it == raw_.end()) return fallback;
    std::string s;
    if (!parseOne(it->second, &s)) throw std::invalid_argument(what + " must be a quoted string.");
    return s;
}

double Params::wallSlipLength() const
{
    const auto it = raw_.find("wallSlipLength");
    if (it == raw_.end()) return 0.0;
    double d;
    if (!parseOne(it->second, &d) || !std::isfinite(d) || d < 0.0)
        throw std::invalid_argument("wallSlipLength must be a finite nonnegative number.");
    return d;
}

const Label& Params::label(std::size_t value) const { return labels_.at(value); }

std::set<std::size_t> Params::labelsOf(unsigned mask) const
{
    std::set<std::size_t> out;
    for (const auto& kv : labels_)
        if (kv.second.type & mask) out.insert(kv.first);
    return out;
}

// FilePrm::ValidateSimulation (fileprm.cpp:136-295), the checks that concern
// the options this engine accepts, with the same messages.
void Params::validate() const
{
    const std::size_t ndim = dimension_.size();
    const std::size_t q = directions();
    if (!((ndim == 2 && q == 9) || (ndim == 3 && q == 19)))
        throw std::invalid_argument("Only D2Q9 and D3Q19 are validated for simulation.");
    std::size_t count = 1;
    for (std::size_t n : dimension_) {
        if (n == 0 || n > std::numeric_limits<std::size_t>::max() / count)
            throw std::invalid_argument("Invalid grid dimensions.");
        count *= n;
    }
    if (fileType() != "uint8") throw std::invalid_argument("Simulation geometry must use uint8 labels.");
    if (tEnd() < tStart() || tEnd() == std::numeric_limits<std::size_t>::max() || tWrite() == 0 ||
        tReport() == 0 || tRestart() == 0)
        throw std::invalid_argument("Invalid time range or zero output/report/restart interval.");
    if (!std::isfinite(stopError()) || stopError() <= 0.0 || !std::isfinite(latticeLen()) || latticeLen() <= 0.0)
        throw std::invalid_argument("Invalid convergence tolerance or lattice length.");
    if (latticeSpeed() != 1.0)
        throw std::invalid_argument("This research implementation requires latticeSpeed=1.");
    const std::string& model = fluidModel();
    if (model != "scsp" && model != "color")
        throw std::invalid_argument("Only scsp and color fluid models are implemented.");
    if (equilModel() != "SRT" && equilModel() != "MRT")
        throw std::invalid_argument("Equilibrium model must be SRT or MRT.");
    const std::size_t phases = model == "color" ? 2 : 1;
    if (relaxationTime_.size() != phases || density_.size() != phases)
        throw std::invalid_argument("Density and relaxation-time counts must match the fluid model.");
    for (std::size_t k = 0; k < phases; ++k)
        if (!std::isfinite(relaxationTime_[k]) || relaxationTime_[k] <= 0.5 ||
            !std::isfinite(density_[k]) || density_[k] <= 0.0)
            throw std::invalid_argument("Densities must be positive; relaxation times must exceed 0.5.");
    // Research selectors: the engine implements the legacy/published-default
    // operators; anything else is refused here instead of silently ignored.
    struct Sel { const char* key; const char* def; };
    const Sel sels[] = {{"wallGradient", "legacy"}, {"viscosityInterpolation", "arithmetic"},
                        {"capillaryModel", "perturbation"}, {"wallRecoloring", "legacy"},
                        {"curvatureStencil", "normal"}, {"phaseBoundary", "bounce"},
                        {"recoloringModel", "cosine"}, {"mrtSpectrum", "legacy"}};
    for (const Sel& s : sels) {
        const std::string v = selector(s.key, s.def, s.key);
        if (v != s.def)
            throw std::invalid_argument(std::string(s.key) + " \"" + v +
                                        "\" is not supported by the B200 engine (only \"" + s.def + "\").");
    }
    if (wallSlipLength() > 0.0)
        throw std::invalid_argument("wallSlipLength is not supported by the B200 engine.");
    if (model == "color") {
        const double a0 = alpha0();
        const double a1 = 1.0 - density_[0] / density_[1] * (1.0 - a0);
        if (!std::isfinite(a0) || a0 < 0.0 || a0 >= 1.0 || !std::isfinite(a1) || a1 < 0.0 || a1 >= 1.0 ||
            !std::isfinite(surfaceTension()) || surfaceTension() < 0.0 ||
            !std::isfinite(interfaceThickness()) || interfaceThickness() < 0.0 || interfaceThickness() > 1.0)
            throw std::invalid_argument("Invalid phase weights, surface tension, or recoloring beta.");
    }
    if (reportDir() >= q) throw std::invalid_argument("Report direction is outside the lattice.");
    if (reportDir() != 0) {
        if (reportSlice_.size() < 2) throw std::invalid_argument("At least two report slices are required.");
        if (*std::max_element(reportSlice_.begin(), reportSlice_.end()) >=
            *std::max_element(dimension_.begin(), dimension_.end()))
            throw std::invalid_argument("Report slice is outside the grid.");
    }
    for (const auto& kv : labels_) {
        if (kv.first > 255) throw std::invalid_argument("Geometry labels must fit in uint8.");
        const Label& v = kv.second;
        if (!std::isfinite(v.value)) throw std::invalid_argument("Non-finite boundary value.");
        if ((v.type == VD || v.type == GV || v.type == PB || v.type == VB || v.type == HF) && v.phase >= phases)
            throw std::invalid_argument("Boundary phase is outside the configured fluid model.");
        if ((v.type == GV || v.type == PB || v.type == VB) && (v.dir == 0 || v.dir >= q))
            throw std::invalid_argument("Boundary direction must be a non-rest lattice direction.");
        if (v.type == PB && v.value <= 0.0)
            throw std::invalid_argument("Pressure-boundary density must be positive.");
        if ((v.type == PB || v.type == VB) && v.dir > 2 * ndim)
            throw std::invalid_argument("Pressure and velocity boundaries require an axial direction.");
        if (v.type == SD && (v.value < 0.0 || v.value > 180.0))
            throw std::invalid_argument("Solid contact angle must be between 0 and 180 degrees.");
        if (v.type == AB) throw std::invalid_argument("Axisymmetric AB boundary handling is not implemented.");
    }
}

}  // namespace lbfhost
