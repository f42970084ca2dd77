// stophys_b200 — command-line host driver over the C ABI.
//
// Mirrors the reference application `StochasticPhysics -parfile:<ini>`
// (Particle_Simulation/Simulator/SimulationApplication.cpp:29-158): read the
// SimulationManagerSettings .ini (Settings/SimulationManagerSettings.h:126-186),
// build every particle through the provider (Provider/ParticleProvider.h:194-217,
// Settings/ParticleSimulationSettings.h:51-152), run the ensemble on the GPU and
// write the mean result {Time, Field, Results, Weight, Mean_Properties}
// (Results/MeanSimulationResult.h:131-141) as JSON, and with Save_single_simulations
// every Save_intervall-th particle's own result (Results/SimulationResultManager.h:115-149).
//
// Accepted keys are the names the reference's serialize() functions use, plus the
// older field layout of its example files (Amplitude_1 = offset, Amplitude_2 =
// excitation, Frequency_1, Phase_1) and the older per-file anisotropy keys
// (Anisotropy_1, Anisotropy_constants_distribution_*).
//
// Usage: stophys_b200 -parfile:<ini> [-sysmatrix:<ini>] [-out:<json>] [-device:N]
//                     [-seed:S] [-precision:fp64|fp32] [-device-provider] [-print]
//   -print parses the files, runs the provider and validates the description
//   without touching a GPU; it writes the description and every particle (with
//   -sysmatrix: the voxels and their offset fields).
//   -device-provider draws the particles on the GPU from the same templates
//   (sp_provider_desc) instead of passing the host-drawn arrays.
//   -sysmatrix runs the system-matrix sweep of the reference
//   (Settings/SystemMatrixSettings.h, Settings/SystemMatrix_SimulationManagerSettings_Factory.h,
//   Simulator/SimulationApplication.cpp:80-128): one ensemble per voxel with the
//   offset field shifted to the voxel's field, all voxels submitted to the
//   continuous-batching server so they share batched launches.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <map>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/stophys_b200.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
    return s;
}

// ------------------------------------------------------------------ .ini
// Sections keep their keys in file order: the provider's particle list is
// ordered as written (ParticleProvider.h:248-267 walks the list in order).
class Ini {
public:
    using Section = std::vector<std::pair<std::string, std::string>>;

    static Ini load(const std::string& path) {
        std::ifstream f(path);
        if (!f) throw std::runtime_error("cannot open " + path);
        Ini ini;
        const auto slash = path.find_last_of('/');
        ini.dir_ = slash == std::string::npos ? "." : path.substr(0, slash);
        std::string line, cur;
        ini.order_.push_back("");
        while (std::getline(f, line)) {
            line = trim(strip_comment(line));
            if (line.empty()) continue;
            if (line.front() == '[' && line.back() == ']') {
                cur = trim(line.substr(1, line.size() - 2));
                if (!ini.sec_.count(cur)) ini.order_.push_back(cur);
                ini.sec_[cur];
                continue;
            }
            const auto eq = line.find('=');
            if (eq == std::string::npos) continue;
            Section& s = ini.sec_[cur];
            const std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
            auto it = std::find_if(s.begin(), s.end(), [&](const auto& kv) { return kv.first == k; });
            if (it == s.end()) s.emplace_back(k, v);
            else it->second = v;  // last assignment wins
        }
        return ini;
    }

    const std::string& dir() const { return dir_; }
    const Section* section(const std::string& s) const {
        auto it = sec_.find(s);
        return it == sec_.end() ? nullptr : &it->second;
    }
    const std::string* find(const std::string& s, const std::string& k) const {
        const Section* sec = section(s);
        if (!sec) return nullptr;
        for (const auto& kv : *sec)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
    // first of the candidate sections that holds the key
    const std::string* any(const std::vector<std::string>& ss, const std::string& k) const {
        for (const auto& s : ss)
            if (auto v = find(s, k)) return v;
        return nullptr;
    }
    // first section, in file order, whose name contains `part` and that holds the key
    const std::string* within(const std::string& part, const std::string& k) const {
        for (const auto& s : order_)
            if (s.find(part) != std::string::npos)
                if (auto v = find(s, k)) return v;
        return nullptr;
    }

    static std::string str(const std::string& v) {
        std::string t = trim(v);
        if (t.size() >= 2 && (t.front() == '\'' || t.front() == '"') && t.back() == t.front()) t = t.substr(1, t.size() - 2);
        return t;
    }
    static double num(const std::string& v) {
        const std::string t = str(v);
        size_t used = 0;
        const double x = std::stod(t, &used);
        if (trim(t.substr(used)).size()) throw std::runtime_error("not a number: '" + v + "'");
        return x;
    }
    static bool boolean(const std::string& v) {
        const std::string t = lower(str(v));
        if (t == "true" || t == "1" || t == "yes") return true;
        if (t == "false" || t == "0" || t == "no") return false;
        throw std::runtime_error("not a boolean: '" + v + "'");
    }
    static std::vector<double> vec(const std::string& v) {
        std::string t = trim(v);
        if (!t.empty() && t.front() == '{') t = t.substr(1);
        if (!t.empty() && t.back() == '}') t.pop_back();
        std::vector<double> out;
        std::stringstream ss(t);
        std::string item;
        while (std::getline(ss, item, ',')) {
            item = trim(item);
            if (!item.empty()) out.push_back(num(item));
        }
        return out;
    }

private:
    std::map<std::string, Section> sec_;
    std::vector<std::string> order_;
    std::string dir_;

    static std::string trim(const std::string& s) {
        const char* ws = " \t\r\n";
        std::string t = s;
        if (t.size() >= 3 && t.compare(0, 3, "\xef\xbb\xbf") == 0) t = t.substr(3);  // UTF-8 byte-order mark
        const auto a = t.find_first_not_of(ws);
        if (a == std::string::npos) return "";
        const auto b = t.find_last_not_of(ws);
        return t.substr(a, b - a + 1);
    }
    // comments: `//`, `%`, `;` and `#` outside quotes
    static std::string strip_comment(const std::string& line) {
        char quote = 0;
        for (size_t i = 0; i < line.size(); ++i) {
            const char c = line[i];
            if (quote) {
                if (c == quote) quote = 0;
                continue;
            }
            if (c == '\'' || c == '"') quote = c;
            else if (c == '%' || c == ';' || c == '#') return line.substr(0, i);
            else if (c == '/' && i + 1 < line.size() && line[i + 1] == '/') return line.substr(0, i);
        }
        return line;
    }
};

// Problem_type / Solver strings of the reference (ProblemSettings.h, SolverSettings.h:39)
int problem_of(const std::string& s) {
    const std::string t = lower(s);
    if (t == "neel") return SP_PROBLEM_NEEL;
    if (t == "neelspherical") return SP_PROBLEM_NEEL_SPHERICAL;
    if (t == "brownandneeleulerspherical") return SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL;
    if (t == "brownandneel") return SP_PROBLEM_BROWN_AND_NEEL;
    throw std::runtime_error("unsupported Problem_type '" + s + "'");
}
int solver_of(const std::string& s) {
    const std::string t = lower(s);
    if (t == "eulermaruyama") return SP_SOLVER_EULER_MARUYAMA;
    if (t == "heun_strong") return SP_SOLVER_HEUN_STRONG;
    if (t == "millstein") return SP_SOLVER_MILLSTEIN;
    if (t == "implicit_midpoint") return SP_SOLVER_IMPLICIT_MIDPOINT;
    if (t == "eulermaruyama_normalized") return SP_SOLVER_EULER_MARUYAMA_NORMALIZED;
    // SolverSettings.cpp:18-20
    if (t == "heun_notconsistent") return SP_SOLVER_HEUN_NOT_CONSISTENT;
    if (t == "weaktest") return SP_SOLVER_WEAK_TEST;
    if (t == "explicitstrong_1.0") return SP_SOLVER_EXPLICIT_STRONG_1;
    throw std::runtime_error("unsupported Solver '" + s + "'");
}

// ------------------------------------------------------------------ provider
// One property distribution of ParticleSimulationSettings.h:62-101 and
// Anisotropy/Uniaxial.hpp:41-85.  With a relative width the draw is
// value * X, X from (1, sigma); otherwise the value itself is drawn around its
// mean.  `sigma_times_mean` selects the radius/shell convention, where an
// absolute width is still scaled by the mean (ParticleSimulationSettings.h:94-101);
// the anisotropy width is an absolute sigma (Uniaxial.hpp:80-84).
// The distribution helper itself lives in an external library the reference
// depends on (MyCEL, not vendored): normal = N(mean, sigma), lognormal with the
// given mean and standard deviation, delta = the mean.
struct Dist {
    std::string type = "delta";
    double width = 0.0;
    bool relative = true;
    bool sigma_times_mean = true;

    double sample(std::mt19937_64& g, double mean, double sigma) const {
        if (type == "delta" || sigma <= 0.0) return mean;
        if (type == "normal") return std::normal_distribution<double>(mean, sigma)(g);
        if (type == "lognormal") {
            const double s2 = std::log1p(sigma * sigma / (mean * mean));
            return std::lognormal_distribution<double>(std::log(mean) - 0.5 * s2, std::sqrt(s2))(g);
        }
        throw std::runtime_error("unsupported distribution type '" + type + "'");
    }
    double apply(std::mt19937_64& g, double value) const {
        if (relative) return value * sample(g, 1.0, width);
        return sample(g, value, sigma_times_mean ? value * width : width);
    }
};

struct ParticleTemplate {
    std::string name, file;
    double count = 0;
    double T = 295, r = 0, Ms = 0, alpha = 0, gamma = 0, K = 0, rh = 0, eta = 0;
    int aniso = SP_ANISOTROPY_UNIAXIAL;
    bool random_orientation = false, random_magnetisation = false;
    double orientation[3] = {0, 0, 0}, magnetisation[3] = {0, 0, 1};
    Dist r_dist, shell_dist, K_dist;
    // uniaxial+cubic (Properties/Anisotropy/UniaxialCubic.hpp): K_cubic, the uniaxial
    // rotation and their distributions
    double K2 = 0, urot[3] = {0, 0, 0};
    Dist K2_dist;
    bool random_urot = false;
};

void read_particle(const Ini& p, ParticleTemplate& t) {
    auto get = [&](const std::string& part, const char* key, double& dst) {
        if (auto v = p.within(part, key)) dst = Ini::num(*v);
    };
    get("Particle_Properties", "Temperature", t.T);
    get("Magnetic_Properties", "Magnetic_radius", t.r);
    get("Magnetic_Properties", "Saturation_magnetisation", t.Ms);
    get("Magnetic_Properties", "Damping_constant", t.alpha);
    get("Magnetic_Properties", "Gyromagnetic_ratio", t.gamma);
    get("Hydrodynamic_Properties", "Hydrodynamic_Radius", t.rh);
    get("Hydrodynamic_Properties", "Viscosity", t.eta);
    if (auto v = p.within("Magnetic_Properties", "Type_of_anisotropy")) {
        const std::string a = lower(Ini::str(*v));
        if (a == "uniaxial") t.aniso = SP_ANISOTROPY_UNIAXIAL;
        else if (a == "cubic") t.aniso = SP_ANISOTROPY_CUBIC;
        else if (a == "uniaxialcubic") t.aniso = SP_ANISOTROPY_UNIAXIAL_CUBIC;
        else throw std::runtime_error("unsupported Type_of_anisotropy '" + a + "'");
    }
    if (t.aniso == SP_ANISOTROPY_UNIAXIAL_CUBIC) {  // UniaxialCubic.hpp:44-50
        if (auto v = p.within("Uniaxial_Part", "K_uniaxial")) t.K = Ini::num(*v);
        else throw std::runtime_error("uniaxialcubic anisotropy needs Uniaxial_Part K_uniaxial");
        if (auto v = p.within("Cubic_Part", "K_cubic")) t.K2 = Ini::num(*v);
        else throw std::runtime_error("uniaxialcubic anisotropy needs Cubic_Part K_cubic");
        if (auto v = p.within("Magnetic_Properties", "Uniaxial_Rotation")) {
            const auto a = Ini::vec(*v);
            if (a.size() != 3) throw std::runtime_error("Uniaxial_Rotation needs three values");
            std::copy(a.begin(), a.end(), t.urot);
        }
    } else {
        const char* kkey = t.aniso == SP_ANISOTROPY_CUBIC ? "K_cubic" : "K_uniaxial";
        if (auto v = p.within("Magnetic_Properties", kkey)) t.K = Ini::num(*v);
        else if (auto v1 = p.within("Magnetic_Properties", "Anisotropy_1")) t.K = Ini::num(*v1);  // older layout
    }

    const std::string init = "Particle_Simulation_Initialization";
    if (auto v = p.within(init, "Use_random_initial_particle_orientation")) t.random_orientation = Ini::boolean(*v);
    if (auto v = p.within(init, "Use_random_initial_particle_magnetisation")) t.random_magnetisation = Ini::boolean(*v);
    auto get3 = [&](const char* key, double* dst) {
        if (auto v = p.within(init, key)) {
            const auto a = Ini::vec(*v);
            if (a.size() != 3) throw std::runtime_error(std::string(key) + " needs three values");
            std::copy(a.begin(), a.end(), dst);
        }
    };
    get3("Initial_particle_orientation", t.orientation);
    get3("Initial_magnetisation_direction", t.magnetisation);

    const std::string ps = "Particle_Simulation_Settings";
    auto read_dist = [&](Dist& d, const char* type, const char* width, const char* rel) {
        if (auto v = p.within(ps, type)) d.type = lower(Ini::str(*v));
        if (auto v = p.within(ps, width)) {
            const auto a = Ini::vec(*v);
            if (!a.empty()) d.width = a[0];
        }
        if (auto v = p.within(ps, rel)) d.relative = Ini::boolean(*v);
    };
    read_dist(t.r_dist, "Magnetic_radius_distribution_type", "Magnetic_radius_distribution_width",
              "Use_relative_distribution_width_for_magnetic_radius");
    read_dist(t.shell_dist, "Hydrodynamic_shell_distribution_type", "Hydrodynamic_shell_distribution_width",
              "Use_relative_distribution_width_for_hydrodynamic_shell");
    t.K_dist.sigma_times_mean = false;
    read_dist(t.K_dist, "Anisotropy_constants_distribution_type", "Anisotropy_constants_distribution_width",
              "Use_relative_distribution_width_for_anisotropy_constants");
    // current layout: [..Anisotropy_Distribution] Distribution_type / Sigma_K_* / Use_relative_distribution_width
    const char* skey = t.aniso == SP_ANISOTROPY_CUBIC ? "Sigma_K_cubic" : "Sigma_K_uniaxial";
    if (t.aniso == SP_ANISOTROPY_UNIAXIAL_CUBIC) {  // UniaxialCubic.hpp:52-88
        auto part = [&](const char* sec, const char* sigma, Dist& d) {
            d.sigma_times_mean = false;
            if (auto v = p.within(sec, sigma)) d.width = Ini::num(*v);
            if (auto v = p.within(sec, "Distribution_type")) d.type = lower(Ini::str(*v));
            if (auto v = p.within(sec, "Use_relative_distribution_width")) d.relative = Ini::boolean(*v);
        };
        part("Uniaxial_Distribution", "Sigma_K_uniaxial", t.K_dist);
        part("Cubic_Distribution", "Sigma_K_cubic", t.K2_dist);
        if (auto v = p.within("Anisotropy_Distribution", "UseRandomCubicOrientation")) t.random_urot = Ini::boolean(*v);
    } else {
        if (auto v = p.within("Anisotropy_Distribution", skey)) t.K_dist.width = Ini::num(*v);
        if (auto v = p.within("Anisotropy_Distribution", "Distribution_type")) t.K_dist.type = lower(Ini::str(*v));
        if (auto v = p.within("Anisotropy_Distribution", "Use_relative_distribution_width")) t.K_dist.relative = Ini::boolean(*v);
    }
}

// Euler angles (ZXZ, psi = 0) whose rotated x axis is the unit vector d: the
// Cartesian Brown problem's state starts at R(phi,theta,psi)·e_x
// (BrownAndNeelRelaxation.inl:295-307), so a random orientation is handed over as
// the angles of a uniformly drawn direction.
void euler_of_direction(const double* d, double* e) {
    const double c = std::max(-1.0, std::min(1.0, d[0]));
    e[0] = std::acos(c);
    e[1] = std::atan2(d[2], -d[1]);
    e[2] = 0.0;
}

struct Run {
    sp_ensemble_desc d{};
    std::vector<double> r, Ms, alpha, gamma, K, rh, eta, euler, mag, K2, urot;
    std::vector<ParticleTemplate> templates;
    std::vector<uint64_t> used;
    std::string savefile;
    // Result_Settings single-simulation keys (ResultSettings.h:90-118)
    bool save_single = false, extra_single_files = false;
    unsigned long long save_interval = 1;
    std::string single_prefix = "Simulation", single_savefile = "ResultsSingle.json";
    bool discrete = false;
    // -device-provider: the templates as an sp_provider_desc (particles drawn on the GPU)
    std::vector<sp_particle_template> dev_templates;
    sp_provider_desc provider{};
};

sp_dist to_sp_dist(const Dist& d) {
    sp_dist o{};
    o.type = d.type == "normal" ? SP_DIST_NORMAL : d.type == "lognormal" ? SP_DIST_LOGNORMAL : SP_DIST_DELTA;
    if (d.type != "normal" && d.type != "lognormal" && d.type != "delta")
        throw std::runtime_error("unsupported distribution type '" + d.type + "'");
    o.relative = d.relative ? 1 : 0;
    o.width = d.width;
    return o;
}

// Hands particle drawing to the device: one sp_particle_template per Particle_List entry
void use_device_provider(Run& run, unsigned long long seed) {
    run.dev_templates.clear();
    for (const auto& t : run.templates) {
        sp_particle_template o{};
        o.weight = t.count;
        o.magnetic_radius = t.r; o.saturation_magnetisation = t.Ms; o.damping_constant = t.alpha;
        o.gyromagnetic_ratio = t.gamma; o.anisotropy_constant = t.K; o.hydrodynamic_radius = t.rh; o.viscosity = t.eta;
        o.cubic_constant = t.K2;
        for (int c = 0; c < 3; ++c) {
            o.orientation[c] = t.orientation[c]; o.magnetisation[c] = t.magnetisation[c]; o.uniaxial_rotation[c] = t.urot[c];
        }
        o.random_orientation = t.random_orientation; o.random_magnetisation = t.random_magnetisation;
        o.random_uniaxial_rotation = t.random_urot;
        o.magnetic_radius_dist = to_sp_dist(t.r_dist);
        o.hydrodynamic_shell_dist = to_sp_dist(t.shell_dist);
        o.anisotropy_dist = to_sp_dist(t.K_dist);
        o.cubic_dist = to_sp_dist(t.K2_dist);
        run.dev_templates.push_back(o);
    }
    run.provider.seed = seed ^ 0xD1B54A32D192ED03ull;
    run.provider.n_templates = static_cast<int32_t>(run.dev_templates.size());
    run.provider.sequential = run.discrete ? 0 : 1;
    run.provider.templates = run.dev_templates.data();
    run.d.provider = &run.provider;
}

Run build(const std::string& path, unsigned long long seed, int precision) {
    const Ini ini = Ini::load(path);
    Run run;
    sp_ensemble_desc& d = run.d;
    d.abi_version = SP_ABI_VERSION;
    d.precision = precision;
    d.noise = SP_NOISE_PHILOX;
    d.seed = seed;
    auto need = [&](const std::string& part, const char* k) -> const std::string& {
        if (auto v = ini.within(part, k)) return *v;
        throw std::runtime_error(std::string("missing key ") + k + " in [" + part + "]");
    };
    auto opt = [&](const std::string& part, const char* k) { return ini.within(part, k); };

    // Simulation_Settings (SimulationSettings.h), Solver_Settings (SolverSettings.h)
    d.timestep = Ini::num(need("Simulation_Settings", "Timestep"));
    d.number_of_steps = static_cast<uint64_t>(Ini::num(need("Simulation_Settings", "Number_of_steps")));
    d.oversampling = static_cast<uint64_t>(Ini::num(need("Simulation_Settings", "Oversampling")));
    d.solver = solver_of(Ini::str(need("Solver_Settings", "Solver")));
    d.max_iteration = opt("Solver_Settings", "Max_Iterations") ? static_cast<int32_t>(Ini::num(*opt("Solver_Settings", "Max_Iterations"))) : 20;
    d.accuracy_goal = opt("Solver_Settings", "Accuracy_Goal") ? Ini::num(*opt("Solver_Settings", "Accuracy_Goal")) : 1e-10;
    // read only for the double-noise solvers (SolverSettings.h:113-116); the default is -1
    d.double_noise_approx = -1;
    if (d.solver == SP_SOLVER_WEAK_TEST || d.solver == SP_SOLVER_EXPLICIT_STRONG_1)
        d.double_noise_approx =
            static_cast<int32_t>(Ini::num(need("Solver_Settings", "Approximation_of_double_noise_integral")));

    // Problem_Settings (ProblemSettings.h:119-206)
    d.problem = problem_of(Ini::str(need("Problem_Settings", "Problem_type")));
    sp_problem_settings& q = d.problem_settings;
    auto pflag = [&](const char* k, int32_t& dst) { if (auto v = opt("Problem_Settings", k)) dst = Ini::boolean(*v); };
    auto pnum = [&](const char* k, double& dst) { if (auto v = opt("Problem_Settings", k)) dst = Ini::num(*v); };
    pflag("Use_coordinate_transformation", q.use_coordinate_transformation);
    pnum("Min_angle_transformation", q.min_angle_before_transformation);
    pnum("Min_angle_before_transformation", q.min_angle_before_transformation);
    pflag("Use_euler_coordinate_transformation", q.use_euler_coordinate_transformation);
    pnum("Brown_Min_angle_before_transformation", q.brown_min_angle_before_transformation);
    pflag("Use_spherical_coordinate_transformation", q.use_spherical_coordinate_transformation);
    pnum("Neel_Min_angle_before_transformation", q.neel_min_angle_before_transformation);
    pflag("Use_simple_model", q.use_simple_model);

    // Field_Properties (FieldProperties.h, Fields/Sinusoidal.hpp:31-34, Fields/Lissajous.hpp:33-36)
    // IFieldMap strings (Fields/FieldList.h:52-60); "zero" accepted beside "none"
    const std::string ft = lower(Ini::str(need("Field_Properties", "Type_of_field")));
    sp_field_desc& f = d.field;
    if (ft == "none" || ft == "zero") f.type = SP_FIELD_ZERO;
    else if (ft == "constant") f.type = SP_FIELD_CONSTANT;
    else if (ft == "sinusoidal") f.type = SP_FIELD_SINUSOIDAL;
    else if (ft == "lissajous") f.type = SP_FIELD_LISSAJOUS;
    else if (ft == "triangular") f.type = SP_FIELD_TRIANGULAR;
    else if (ft == "rectangular") f.type = SP_FIELD_RECTANGULAR;
    else if (ft == "sinc") f.type = SP_FIELD_SINC;
    else throw std::runtime_error("unsupported Type_of_field '" + ft + "'");
    auto put3 = [](double* dst, const std::vector<double>& v, const char* k) {
        if (v.size() != 3) throw std::runtime_error(std::string(k) + " needs three values");
        std::copy(v.begin(), v.end(), dst);
    };
    auto fvec = [&](const char* k, double* dst) {
        if (auto v = opt("Field_Properties", k)) { put3(dst, Ini::vec(*v), k); return true; }
        return false;
    };
    auto fnum = [&](const char* k, double* dst) {
        if (auto v = opt("Field_Properties", k)) { *dst = Ini::num(*v); return true; }
        return false;
    };
    if (!fvec("Offset_Field", f.offset)) fvec("Amplitude_1", f.offset);
    if (!fvec("Amplitude", f.amplitude)) fvec("Amplitude_2", f.amplitude);
    if (!fvec("Frequencies", f.frequency) && !fnum("Frequency", f.frequency)) fnum("Frequency_1", f.frequency);
    if (!fvec("Phases", f.phase) && !fnum("Phase", f.phase)) fnum("Phase_1", f.phase);
    // Fields/Triangular.hpp, Rectangular.hpp, Sinc.hpp
    fnum("Periode", &f.periode);
    fnum("TimeOffset", &f.time_offset);
    fnum("Tau", &f.tau);
    if (auto v = opt("Field_Properties", "Alternating")) f.alternating = Ini::boolean(*v);

    // Particle_Provider (ParticleProvider.h:243-292)
    bool discrete = false;
    if (auto v = opt("Particle_Provider", "Use_discrete_distribution_to_select_particle")) discrete = Ini::boolean(*v);
    run.discrete = discrete;
    const Ini::Section* list = ini.section("Particle_Provider.Particle_List");
    if (!list || list->empty()) throw std::runtime_error("no [Particle_Provider.Particle_List]");
    for (const auto& kv : *list) {
        ParticleTemplate t;
        t.name = kv.first;
        t.file = Ini::str(kv.second);
        const std::string* c = ini.find("Particle_Provider.Particle_Numbers", kv.first);
        if (!c) throw std::runtime_error("no Particle_Numbers entry for " + kv.first);
        t.count = Ini::num(*c);
        if (!t.file.empty()) {
            const std::string fp = t.file.front() == '/' ? t.file : ini.dir() + "/" + t.file;
            read_particle(Ini::load(fp), t);
        } else {
            read_particle(ini, t);  // properties stored under the particle's name in the same file
        }
        run.templates.push_back(t);
    }
    run.used.assign(run.templates.size(), 0);
    const uint64_t n = static_cast<uint64_t>(Ini::num(need("Simulation_Settings", "Number_of_simulations")));
    d.temperature = run.templates[0].T;
    d.anisotropy = run.templates[0].aniso;
    for (const auto& t : run.templates)
        if (t.aniso != d.anisotropy || t.T != d.temperature)
            throw std::runtime_error("all particles of one run must share temperature and type of anisotropy");

    std::mt19937_64 g(seed ^ 0x9E3779B97F4A7C15ull);
    std::vector<double> weights;
    for (const auto& t : run.templates) weights.push_back(t.count);
    std::discrete_distribution<size_t> pick(weights.begin(), weights.end());
    std::uniform_real_distribution<double> u(0.0, 1.0);
    std::normal_distribution<double> z(0.0, 1.0);
    for (uint64_t i = 0; i < n; ++i) {
        size_t k = 0;
        if (discrete) {
            k = pick(g);
            ++run.used[k];
        } else {  // fill each template's count in list order; past the total, the first,
                  // uncounted (ParticleProvider.h:201-213)
            for (size_t c = 0; c < run.templates.size(); ++c)
                if (run.used[c] < run.templates[c].count) {
                    k = c;
                    ++run.used[c];
                    break;
                }
        }
        const ParticleTemplate& p = run.templates[k];
        // applySettingsToParticleProperties order: anisotropy, radius, then the shell
        // around the new radius (ParticleSimulationSettings.h:138-144, 78-92)
        const double K = p.K_dist.apply(g, p.K);
        if (d.anisotropy == SP_ANISOTROPY_UNIAXIAL_CUBIC) {
            run.K2.push_back(p.K2_dist.apply(g, p.K2));
            double ur[3] = {p.urot[0], p.urot[1], p.urot[2]};
            if (p.random_urot) {  // UniaxialCubic.hpp:66-75: U[0,2pi), U[0,pi), U[0,2pi)
                ur[0] = u(g) * 2 * kPi; ur[1] = u(g) * kPi; ur[2] = u(g) * 2 * kPi;
            }
            for (double c : ur) run.urot.push_back(c);
        }
        const double r = p.r_dist.apply(g, p.r);
        const double rh = p.shell_dist.apply(g, p.rh - r) + r;
        run.K.push_back(K); run.r.push_back(r); run.rh.push_back(rh);
        run.Ms.push_back(p.Ms); run.alpha.push_back(p.alpha); run.gamma.push_back(p.gamma); run.eta.push_back(p.eta);

        double e[3] = {p.orientation[0], p.orientation[1], p.orientation[2]};
        double m[3] = {p.magnetisation[0], p.magnetisation[1], p.magnetisation[2]};
        const bool cartesian = d.problem == SP_PROBLEM_NEEL || d.problem == SP_PROBLEM_BROWN_AND_NEEL;
        if (p.random_orientation) {
            if (d.problem == SP_PROBLEM_NEEL) {  // NeelRelaxation.h:226-235: all three angles U[0, 2pi)
                for (double& c : e) c = u(g) * 2 * kPi;
            } else if (d.problem == SP_PROBLEM_BROWN_AND_NEEL) {  // BrownAndNeelRelaxation.inl:288-294
                double dir[3] = {z(g), z(g), z(g)};
                const double nd = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
                for (double& c : dir) c /= nd;
                euler_of_direction(dir, e);
            } else {  // ParticleStateInitializer.h:50-56
                e[0] = u(g) * 2 * kPi; e[1] = u(g) * kPi; e[2] = u(g) * 2 * kPi;
            }
        }
        if (p.random_magnetisation) {
            if (cartesian) {  // NeelRelaxation.h:268-283, BrownAndNeelRelaxation.inl:309-315
                for (double& c : m) c = z(g);
            } else {  // ParticleStateInitializer.h:113-123
                const double ph = u(g) * 2 * kPi, th = u(g) * kPi;
                m[0] = std::cos(ph) * std::sin(th); m[1] = std::sin(ph) * std::sin(th); m[2] = std::cos(th);
            }
        }
        const double nm = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        if (!(nm > 0)) throw std::runtime_error("initial magnetisation direction is zero");
        for (int c = 0; c < 3; ++c) { run.euler.push_back(e[c]); run.mag.push_back(m[c] / nm); }
    }
    d.n_particles = n;
    const bool uc = d.anisotropy == SP_ANISOTROPY_UNIAXIAL_CUBIC;
    d.particles = {run.r.data(), run.Ms.data(), run.alpha.data(), run.gamma.data(), run.K.data(),
                   run.rh.data(), run.eta.data(), run.euler.data(), run.mag.data(),
                   uc ? run.K2.data() : nullptr, uc ? run.urot.data() : nullptr};
    if (auto v = opt("Result_Settings", "Savefile")) run.savefile = Ini::str(*v);
    if (auto v = opt("Result_Settings", "Save_single_simulations")) run.save_single = Ini::boolean(*v);
    if (auto v = opt("Result_Settings", "Use_extra_file_for_single_simulations")) run.extra_single_files = Ini::boolean(*v);
    if (auto v = opt("Result_Settings", "Save_single_name_prefix")) run.single_prefix = Ini::str(*v);
    if (auto v = opt("Result_Settings", "Single_simulations_savefile")) run.single_savefile = Ini::str(*v);
    if (auto v = opt("Result_Settings", "Save_intervall")) {
        const double iv = Ini::num(*v);
        if (!(iv >= 1) || iv != std::floor(iv)) throw std::runtime_error("Save_intervall must be a positive integer");
        run.save_interval = static_cast<unsigned long long>(iv);
    }
    return run;
}

// ------------------------------------------------------------------ single-simulation results
// SimulationResultManager::addSingleResult (Results/SimulationResultManager.h:115-149):
// result counter c = 1, 2, ... (particle order here; completion order in the reference's
// thread pool); every Save_intervall-th is written as the named value <prefix>_<c>, either
// all into Single_simulations_savefile or, with Use_extra_file_for_single_simulations, each
// into its own file named <prefix>_<c> beside it with its extension.  The reference refuses
// a single-results file equal to Savefile.  Files are JSON (the reference's SerAr MATLAB/HDF5
// archives are not available), so a configured extension other than .json becomes .json.
std::string json_path(const std::string& path) {
    const auto slash = path.find_last_of('/');
    const auto dot = path.find_last_of('.');
    const bool has_ext = dot != std::string::npos && (slash == std::string::npos || dot > slash);
    return (has_ext ? path.substr(0, dot) : path) + ".json";
}
std::string single_name(const Run& run, unsigned long long counter) {
    return run.single_prefix + "_" + std::to_string(counter);
}
std::string single_file(const Run& run, unsigned long long counter) {
    const std::string base = json_path(run.single_savefile);
    if (!run.extra_single_files) return base;
    const auto slash = base.find_last_of('/');
    const std::string dir = slash == std::string::npos ? "" : base.substr(0, slash + 1);
    return dir + single_name(run, counter) + ".json";
}
// number of particles the single-result settings select (counter % interval == 0)
unsigned long long single_count(const Run& run) {
    return run.save_single ? run.d.n_particles / run.save_interval : 0;
}
void check_single_settings(const Run& run) {
    if (single_count(run) > 0 && run.single_savefile == run.savefile)
        throw std::runtime_error("Writing SingleResults and MeanResult to same file currently not supported!");
}

// ------------------------------------------------------------------ system matrix
// [System_Matrix_Settings] Startfield, Stopfield, Slices, Use_start_stop_Voxel,
// Start_Voxel, Stop_Voxel (SystemMatrixSettings.h:276-303)
struct SysMat {
    double start[3] = {0, 0, 0}, stop[3] = {1, 1, 1};
    unsigned long long slices[3] = {0, 0, 0}, vstart[3] = {0, 0, 0}, vstop[3] = {1, 1, 1};
    bool use_start_stop = false;

    static SysMat load(const std::string& path) {
        const Ini ini = Ini::load(path);
        SysMat m;
        auto vec3 = [&](const char* k, double* dst, bool required) {
            const std::string* v = ini.within("System_Matrix_Settings", k);
            if (!v) {
                if (required) throw std::runtime_error(std::string("missing key ") + k + " in [System_Matrix_Settings]");
                return;
            }
            const auto a = Ini::vec(*v);
            if (a.size() != 3) throw std::runtime_error(std::string(k) + " needs three values");
            std::copy(a.begin(), a.end(), dst);
        };
        auto idx3 = [&](const char* k, unsigned long long* dst, bool required) {
            double t[3] = {0, 0, 0};
            vec3(k, t, required);
            for (int i = 0; i < 3; ++i) {
                if (t[i] < 0 || t[i] != std::floor(t[i])) throw std::runtime_error(std::string(k) + " must hold non-negative integers");
                dst[i] = static_cast<unsigned long long>(t[i]);
            }
        };
        vec3("Startfield", m.start, true);
        vec3("Stopfield", m.stop, true);
        idx3("Slices", m.slices, true);
        if (auto v = ini.within("System_Matrix_Settings", "Use_start_stop_Voxel")) m.use_start_stop = Ini::boolean(*v);
        for (int i = 0; i < 3; ++i) {
            if (m.slices[i] < 1) throw std::runtime_error("SystemMatrixSettings: Number of Voxels must be at least one for every dimension!");
            // a single slice needs Startfield == Stopfield in that direction (:52-76)
            if (m.slices[i] == 1 && std::abs(m.stop[i] - m.start[i]) > 1e-15 * std::max(1.0, std::abs(m.stop[i])))
                throw std::runtime_error("SystemMatrixSettings: Invalid Parameters. Unable to calculate VoxelSize.");
        }
        if (m.use_start_stop) {
            idx3("Start_Voxel", m.vstart, true);
            idx3("Stop_Voxel", m.vstop, true);
            for (int i = 0; i < 3; ++i)
                if (m.vstart[i] > m.slices[i] || m.vstop[i] > m.slices[i])
                    throw std::runtime_error("SystemMatrixSettings: Start/Stop voxel beyond the defined slices");
        } else {
            for (int i = 0; i < 3; ++i) { m.vstart[i] = 0; m.vstop[i] = m.slices[i] - 1; }
        }
        return m;
    }
    // Size_FOV / max(slices - 1, 1) per direction (:247-268)
    void voxel_size(double* out) const {
        for (int i = 0; i < 3; ++i)
            out[i] = (stop[i] - start[i]) / static_cast<double>(slices[i] > 1 ? slices[i] - 1 : 1);
    }
    // getNumberVoxelsToSimulate (:159-182), including its signed-difference rule
    unsigned long long count() const {
        if (!use_start_stop) return slices[0] * slices[1] * slices[2];
        auto absdiff = [](unsigned long long a, unsigned long long b) { return a > b ? a - b : b - a; };
        const unsigned long long zp = absdiff(vstart[2], vstop[2]) * slices[0] * slices[1];
        const unsigned long long yp = absdiff(vstart[1], vstop[1]) * slices[0];
        const unsigned long long xp = absdiff(vstart[0], vstop[0]);
        return vstart[0] > vstop[0] ? yp + zp - xp : xp + yp + zp;
    }
    // generateSimulationVoxels (:184-215): z-major from the start voxel, x fastest
    std::vector<std::array<unsigned long long, 3>> voxels() const {
        std::vector<std::array<unsigned long long, 3>> out;
        const unsigned long long n = count();
        unsigned long long sv[3] = {vstart[0], vstart[1], vstart[2]};
        for (unsigned long long z = sv[2]; z < slices[2] && out.size() < n; ++z) {
            for (unsigned long long y = sv[1]; y < slices[1] && out.size() < n; ++y) {
                for (unsigned long long x = sv[0]; x < slices[0] && out.size() < n; ++x) out.push_back({x, y, z});
                sv[0] = 0;
            }
            sv[1] = 0;
        }
        return out;
    }
};

// ------------------------------------------------------------------ JSON
std::string jnum(double v) {
    if (!std::isfinite(v)) return "null";
    char b[40];
    std::snprintf(b, sizeof(b), "%.17g", v);
    return b;
}
std::string jstr(const std::string& s) {
    std::string o = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o + "\"";
}
void jarr(std::ostream& o, const double* v, size_t n) {
    o << "[";
    for (size_t i = 0; i < n; ++i) o << (i ? "," : "") << jnum(v[i]);
    o << "]";
}
void jrows(std::ostream& o, const double* v, size_t rows, size_t cols) {
    o << "[";
    for (size_t r = 0; r < rows; ++r) {
        if (r) o << ",";
        jarr(o, v + r * cols, cols);
    }
    o << "]";
}
double mean_of(const std::vector<double>& v) {
    double s = 0;
    for (double x : v) s += x;
    return v.empty() ? 0.0 : s / static_cast<double>(v.size());
}

void write_description(std::ostream& o, const Run& run) {
    const sp_ensemble_desc& d = run.d;
    const sp_problem_settings& q = d.problem_settings;
    const size_t n = d.n_particles;
    o << "{\"problem\":" << d.problem << ",\"solver\":" << d.solver << ",\"anisotropy\":" << d.anisotropy
      << ",\"precision\":" << d.precision << ",\"n_particles\":" << n << ",\"number_of_steps\":" << d.number_of_steps
      << ",\"oversampling\":" << d.oversampling << ",\"timestep\":" << jnum(d.timestep)
      << ",\"temperature\":" << jnum(d.temperature) << ",\"max_iteration\":" << d.max_iteration
      << ",\"accuracy_goal\":" << jnum(d.accuracy_goal) << ",\"double_noise_approx\":" << d.double_noise_approx
      << ",\"field\":{\"type\":" << d.field.type << ",\"offset\":";
    jarr(o, d.field.offset, 3);
    o << ",\"amplitude\":";
    jarr(o, d.field.amplitude, 3);
    o << ",\"frequency\":";
    jarr(o, d.field.frequency, 3);
    o << ",\"phase\":";
    jarr(o, d.field.phase, 3);
    o << ",\"periode\":" << jnum(d.field.periode) << ",\"time_offset\":" << jnum(d.field.time_offset)
      << ",\"tau\":" << jnum(d.field.tau) << ",\"alternating\":" << d.field.alternating;
    o << "},\"problem_settings\":{\"use_coordinate_transformation\":" << q.use_coordinate_transformation
      << ",\"min_angle_before_transformation\":" << jnum(q.min_angle_before_transformation)
      << ",\"use_euler_coordinate_transformation\":" << q.use_euler_coordinate_transformation
      << ",\"brown_min_angle_before_transformation\":" << jnum(q.brown_min_angle_before_transformation)
      << ",\"use_spherical_coordinate_transformation\":" << q.use_spherical_coordinate_transformation
      << ",\"neel_min_angle_before_transformation\":" << jnum(q.neel_min_angle_before_transformation)
      << ",\"use_simple_model\":" << q.use_simple_model << "},\"used_particle_numbers\":{";
    for (size_t k = 0; k < run.templates.size(); ++k)
        o << (k ? "," : "") << jstr(run.templates[k].name) << ":" << run.used[k];
    o << "},\"particles\":{\"magnetic_radius\":";
    jarr(o, run.r.data(), n);
    o << ",\"saturation_magnetisation\":";
    jarr(o, run.Ms.data(), n);
    o << ",\"damping_constant\":";
    jarr(o, run.alpha.data(), n);
    o << ",\"gyromagnetic_ratio\":";
    jarr(o, run.gamma.data(), n);
    o << ",\"anisotropy_constant\":";
    jarr(o, run.K.data(), n);
    o << ",\"hydrodynamic_radius\":";
    jarr(o, run.rh.data(), n);
    o << ",\"viscosity\":";
    jarr(o, run.eta.data(), n);
    o << ",\"orientation\":";
    jrows(o, run.euler.data(), n, 3);
    o << ",\"magnetisation\":";
    jrows(o, run.mag.data(), n, 3);
    if (d.anisotropy == SP_ANISOTROPY_UNIAXIAL_CUBIC) {
        o << ",\"cubic_constant\":";
        jarr(o, run.K2.data(), n);
        o << ",\"uniaxial_rotation\":";
        jrows(o, run.urot.data(), n, 3);
    }
    o << "},\"single_results\":[";
    for (unsigned long long i = 0; i < single_count(run); ++i) {
        const unsigned long long c = (i + 1) * run.save_interval;
        o << (i ? "," : "") << "{\"particle\":" << c - 1 << ",\"name\":" << jstr(single_name(run, c))
          << ",\"file\":" << jstr(single_file(run, c)) << "}";
    }
    o << "],\"savefile\":" << jstr(run.savefile) << "}\n";
}

void write_mean_results(std::ostream& os, const std::vector<double>& time, const std::vector<double>& field,
                        const std::vector<double>& mean, const std::vector<double>& weight, size_t K, size_t od,
                        const Run& run) {
    const sp_ensemble_desc& d = run.d;
    os << "{\"Time\":";
    jarr(os, time.data(), K);
    os << ",\"Field\":";
    jrows(os, field.data(), K, 3);
    os << ",\"Results\":";
    jrows(os, mean.data(), K, od);
    os << ",\"Weight\":";
    jarr(os, weight.data(), od);
    os << ",\"Mean_Properties\":{\"Temperature\":" << jnum(d.temperature)
       << ",\"Magnetic_radius\":" << jnum(mean_of(run.r)) << ",\"Saturation_magnetisation\":" << jnum(mean_of(run.Ms))
       << ",\"Damping_constant\":" << jnum(mean_of(run.alpha)) << ",\"Gyromagnetic_ratio\":" << jnum(mean_of(run.gamma))
       << ",\"Anisotropy_constant\":" << jnum(mean_of(run.K)) << ",\"Hydrodynamic_Radius\":" << jnum(mean_of(run.rh))
       << ",\"Viscosity\":" << jnum(mean_of(run.eta)) << "}}";
}

// The recorded window means of the selected particles, one named value each
// (SingleSimulationResult::save, Results/SingleSimulationResult.h:96-104: UsedProperties,
// Time, Weight, Field, Results).  traj is [count][K][od] as sp_result returns it.
void write_single_results(const Run& run, const std::vector<double>& traj, const std::vector<double>& time,
                          const std::vector<double>& field, size_t K, size_t od) {
    const sp_ensemble_desc& d = run.d;
    const unsigned long long count = single_count(run);
    std::ofstream shared;
    for (unsigned long long i = 0; i < count; ++i) {
        const unsigned long long c = (i + 1) * run.save_interval, p = c - 1;
        std::ofstream own;
        std::ofstream& f = run.extra_single_files ? own : shared;
        if (run.extra_single_files || i == 0) {
            f.open(single_file(run, c));
            if (!f) throw std::runtime_error("cannot write " + single_file(run, c));
            f << "{";
        } else {
            f << ",";
        }
        // getWeighting: Ms V for every output, 1 for the axis of the coupled Cartesian problem
        // (NeelRelaxation.h:287-291, BrownAndNeelRelaxation.h:152-159)
        const double kPi = 3.14159265358979323846;
        const double moment = run.Ms[p] * 4.0 / 3.0 * kPi * run.r[p] * run.r[p] * run.r[p];
        std::vector<double> w(od, moment);
        if (d.problem == SP_PROBLEM_BROWN_AND_NEEL)
            for (size_t k = 0; k < 3; ++k) w[k] = 1.0;
        f << jstr(single_name(run, c)) << ":{\"UsedProperties\":{\"Temperature\":" << jnum(d.temperature)
          << ",\"Magnetic_radius\":" << jnum(run.r[p]) << ",\"Saturation_magnetisation\":" << jnum(run.Ms[p])
          << ",\"Damping_constant\":" << jnum(run.alpha[p]) << ",\"Gyromagnetic_ratio\":" << jnum(run.gamma[p])
          << ",\"Anisotropy_constant\":" << jnum(run.K[p]) << ",\"Hydrodynamic_Radius\":" << jnum(run.rh[p])
          << ",\"Viscosity\":" << jnum(run.eta[p]) << "},\"Time\":";
        jarr(f, time.data(), K);
        f << ",\"Weight\":";
        jarr(f, w.data(), od);
        f << ",\"Field\":";
        jrows(f, field.data(), K, 3);
        f << ",\"Results\":";
        jrows(f, traj.data() + i * K * od, K, od);
        f << "}";
        if (run.extra_single_files || i + 1 == count) {
            f << "}\n";
            f.close();
            if (!f) throw std::runtime_error("writing " + single_file(run, c) + " failed");
        }
    }
}

// File name of one voxel's result: Savefile stem + "_Vox_x_y_z" + extension
// (SystemMatrix_SimulationManagerSettings_Factory.h:44-63)
std::string voxel_file(const std::string& savefile, const std::array<unsigned long long, 3>& v) {
    const std::string base = savefile.empty() ? "Result.json" : savefile;
    const auto slash = base.find_last_of('/');
    const auto dot = base.find_last_of('.');
    const bool has_ext = dot != std::string::npos && (slash == std::string::npos || dot > slash);
    const std::string stem = has_ext ? base.substr(0, dot) : base, ext = has_ext ? base.substr(dot) : "";
    return stem + "_Vox_" + std::to_string(v[0]) + "_" + std::to_string(v[1]) + "_" + std::to_string(v[2]) + ext;
}

// One ensemble per voxel: the base description with the offset field moved to
// Startfield + VoxelSize * voxel (added to the configured offset, :36-42) and its
// own Philox key (seed + voxel number), all submitted to one server.
int run_sysmatrix(const Run& run, const SysMat& sm, std::ostream& os, int device, bool print_only) {
    const auto vox = sm.voxels();
    double size[3];
    sm.voxel_size(size);
    std::vector<sp_ensemble_desc> descs;
    for (size_t i = 0; i < vox.size(); ++i) {
        sp_ensemble_desc d = run.d;
        for (int c = 0; c < 3; ++c)
            d.field.offset[c] = run.d.field.offset[c] + sm.start[c] + size[c] * static_cast<double>(vox[i][c]);
        d.seed = run.d.seed + i;
        descs.push_back(d);
    }
    auto write_header = [&]() {
        os << "{\"System_Matrix_Settings\":{\"Startfield\":";
        jarr(os, sm.start, 3);
        os << ",\"Stopfield\":";
        jarr(os, sm.stop, 3);
        os << ",\"Slices\":[" << sm.slices[0] << "," << sm.slices[1] << "," << sm.slices[2]
           << "],\"Use_start_stop_Voxel\":" << (sm.use_start_stop ? "true" : "false") << ",\"Start_Voxel\":["
           << sm.vstart[0] << "," << sm.vstart[1] << "," << sm.vstart[2] << "],\"Stop_Voxel\":[" << sm.vstop[0] << ","
           << sm.vstop[1] << "," << sm.vstop[2] << "],\"Voxel_Size\":";
        jarr(os, size, 3);
        os << "},\"Number_of_voxels\":" << vox.size() << ",\"Voxels\":[";
    };
    write_header();
    if (print_only) {
        for (size_t i = 0; i < vox.size(); ++i) {
            os << (i ? "," : "") << "{\"Voxel\":[" << vox[i][0] << "," << vox[i][1] << "," << vox[i][2]
               << "],\"Offset_Field\":";
            jarr(os, descs[i].field.offset, 3);
            os << ",\"Seed\":" << descs[i].seed << ",\"File\":" << jstr(voxel_file(run.savefile, vox[i])) << "}";
        }
        os << "]}\n";
        return 0;
    }
    sp_context* ctx = nullptr;
    if (sp_create(&ctx, device) != SP_OK) throw std::runtime_error(sp_last_error());
    sp_server* srv = nullptr;
    sp_server_config cfg{};
    if (sp_server_create(ctx, &cfg, &srv) != SP_OK) {
        sp_destroy(ctx);
        throw std::runtime_error(sp_last_error());
    }
    std::vector<uint64_t> ids(descs.size());
    std::string err;
    for (size_t i = 0; i < descs.size() && err.empty(); ++i)
        if (sp_server_submit(srv, &descs[i], &ids[i]) != SP_OK) err = sp_last_error();
    int32_t sd = 0, nd = 0, od = 0;
    sp_query_dims(run.d.problem, &sd, &nd, &od);
    const size_t K = run.d.number_of_steps / run.d.oversampling;
    uint64_t total_steps = 0;
    double max_latency = 0.0;
    for (size_t i = 0; i < descs.size() && err.empty(); ++i) {
        std::vector<double> mean(K * od), weight(od), time(K), field(3 * K);
        sp_result res{mean.data(), weight.data(), time.data(), field.data(), nullptr, nullptr, nullptr};
        sp_stats st{};
        double lat = 0.0;
        if (sp_server_wait(srv, ids[i], -1.0, &res, &st, &lat) != SP_OK) {
            err = sp_last_error();
            break;
        }
        total_steps += st.particle_steps;
        max_latency = std::max(max_latency, lat);
        os << (i ? "," : "") << "{\"Voxel\":[" << vox[i][0] << "," << vox[i][1] << "," << vox[i][2]
           << "],\"Offset_Field\":";
        jarr(os, descs[i].field.offset, 3);
        os << ",\"File\":" << jstr(voxel_file(run.savefile, vox[i])) << ",\"Mean_Results\":";
        write_mean_results(os, time, field, mean, weight, K, static_cast<size_t>(od), run);
        os << "}";
    }
    sp_server_destroy(srv);
    sp_destroy(ctx);
    if (!err.empty()) throw std::runtime_error(err);
    os << "],\"Stats\":{\"particle_steps\":" << total_steps << ",\"max_latency_ms\":" << jnum(max_latency) << "}}\n";
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    std::string par, out, sysmatrix;
    int device = 0, precision = SP_PRECISION_FP64;
    unsigned long long seed = 0x5EED;
    bool print_only = false, device_provider = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&](const char* p) { return a.substr(std::string(p).size()); };
        if (a.rfind("-parfile:", 0) == 0) par = val("-parfile:");
        else if (a.rfind("-out:", 0) == 0) out = val("-out:");
        else if (a.rfind("-sysmatrix:", 0) == 0) sysmatrix = val("-sysmatrix:");
        else if (a.rfind("-device:", 0) == 0) device = std::atoi(val("-device:").c_str());
        else if (a.rfind("-seed:", 0) == 0) seed = std::strtoull(val("-seed:").c_str(), nullptr, 0);
        else if (a == "-precision:fp32") precision = SP_PRECISION_FP32;
        else if (a == "-precision:fp64") precision = SP_PRECISION_FP64;
        else if (a == "-print") print_only = true;
        else if (a == "-device-provider") device_provider = true;
        else {
            std::fprintf(stderr, "unknown argument %s\n", a.c_str());
            return 2;
        }
    }
    if (par.empty()) {
        std::fprintf(stderr, "usage: stophys_b200 -parfile:<ini> [-sysmatrix:<ini>] [-out:<json>] [-device:N] "
                             "[-seed:S] [-precision:fp64|fp32] [-device-provider] [-print]\n");
        return 2;
    }
    try {
        Run run = build(par, seed, precision);
        if (device_provider && !print_only) use_device_provider(run, seed);
        const sp_ensemble_desc& d = run.d;
        if (sp_validate(&d) != SP_OK) throw std::runtime_error(sp_last_error());
        std::ofstream fo;
        if (!out.empty()) {
            fo.open(out);
            if (!fo) throw std::runtime_error("cannot write " + out);
        }
        std::ostream& os = out.empty() ? std::cout : fo;
        check_single_settings(run);
        if (!sysmatrix.empty()) {
            if (single_count(run) > 0)
                std::fprintf(stderr, "stophys_b200: Save_single_simulations applies to plain runs; the system-matrix "
                                     "sweep writes mean results only\n");
            return run_sysmatrix(run, SysMat::load(sysmatrix), os, device, print_only);
        }
        if (print_only) {
            write_description(os, run);
            return 0;
        }
        int32_t sd = 0, nd = 0, od = 0;
        if (sp_query_dims(d.problem, &sd, &nd, &od) != SP_OK) throw std::runtime_error(sp_last_error());
        const size_t K = d.number_of_steps / d.oversampling;
        std::vector<double> mean(K * od), weight(od), time(K), field(3 * K);
        sp_result res{mean.data(), weight.data(), time.data(), field.data(), nullptr, nullptr, nullptr};
        // single-simulation results: the device records every Save_intervall-th particle only
        const unsigned long long nsingle = single_count(run);
        std::vector<double> traj;
        if (nsingle > 0) {
            if (run.save_interval > 0x7fffffffull) throw std::runtime_error("Save_intervall exceeds 2^31 - 1");
            run.d.record_trajectories = static_cast<int32_t>(run.save_interval);
            traj.assign(nsingle * K * od, 0.0);
            res.trajectories = traj.data();
        }
        sp_stats st{};
        sp_context* ctx = nullptr;
        if (sp_create(&ctx, device) != SP_OK) throw std::runtime_error(sp_last_error());
        const sp_status s = sp_simulate(ctx, &d, &res, &st);
        if (s == SP_OK && d.provider) {  // Mean_Properties of the particles the device drew
            std::vector<double> p(20 * d.n_particles);
            if (sp_provide_particles(ctx, &d, p.data()) != SP_OK) {
                sp_destroy(ctx);
                throw std::runtime_error(sp_last_error());
            }
            for (auto* v : {&run.r, &run.Ms, &run.alpha, &run.gamma, &run.K, &run.rh, &run.eta}) v->assign(d.n_particles, 0.0);
            for (size_t i = 0; i < d.n_particles; ++i) {
                const double* o = p.data() + 20 * i;
                run.r[i] = o[0]; run.Ms[i] = o[1]; run.alpha[i] = o[2]; run.gamma[i] = o[3]; run.K[i] = o[4];
                run.rh[i] = o[5]; run.eta[i] = o[6];
            }
        }
        sp_destroy(ctx);
        if (s != SP_OK) throw std::runtime_error(sp_last_error());
        if (nsingle > 0) write_single_results(run, traj, time, field, K, static_cast<size_t>(od));
        os << "{\"Mean_Results\":";
        write_mean_results(os, time, field, mean, weight, K, static_cast<size_t>(od), run);
        os << ",\"Stats\":{\"particle_steps\":" << st.particle_steps
           << ",\"nonfinite_particles\":" << st.nonfinite_particles << ",\"device_ms\":" << jnum(st.device_ms)
           << "},\"Savefile\":" << jstr(run.savefile) << "}\n";
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "stophys_b200: %s\n", e.what());
        return 1;
    }
}
