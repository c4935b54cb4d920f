// deck.hpp -- the reader of a Schemi task deck (set/*.txt), shared by the task-deck driver fvrun
// and the step-solver adapter that runs inside the reference's own main.
//
// Reads what the reference reads (paths inside the Schemi project): set/g.txt and set/main.txt
// (the 24 positional keys of main/Schemi.cpp:83-163), set/zonesDescription.txt (zone.cpp),
// set/sub_<k>.txt, set/velocity.txt, set/pressure.txt (phaseInitialization.cpp), the EOS data
// files of abstractMixtureThermodynamics.cpp and set/chemicalKinetics.txt, with the reference's
// stream extraction and its messages, into an fv_config and the zone values of a fresh run.
#pragma once

#include <algorithm>
#include <cmath>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "fvstep.h"

namespace fvdeck {

constexpr double kNA = 6.02214076E23;          // globalConstants.hpp NAvogardro
constexpr double kRSI = 8.31446261815324;      // R_SI
constexpr double kPlanckSI = 6.626E-34;        // PlanckConstant_SI
inline const double kPi = std::acos(-1.0);            // Pi_number (g++ build)
constexpr double kStab = 5 * 2.220446049250313080847e-16;  // stabilizator
constexpr int kPrecision = 20;                 // ioPrecision
constexpr int kNumberLength = 6;               // lengthOfNumber

struct Fail : std::runtime_error {
    int code;
    Fail(const std::string& m, int c = FV_ERR_INIT) : std::runtime_error(m), code(c) {}
};

// A file read by the same stream extractions as the reference's operator>> chains: a string is
// the next whitespace-delimited word, a number the longest prefix that parses as a double and no
// more, so "0;" yields 0 and leaves ";" for the next word (zone.cpp:64-65 reads the shipped
// "1 0 0; 0.5 0.5 0.5" plane this way).
struct Tokens {
    std::istringstream in;
    Tokens(const std::string& path) {
        std::ifstream f(path);
        if (!f.is_open()) throw Fail(path + " not found.", FV_ERR_SYSTEM);
        std::ostringstream all;
        all << f.rdbuf();
        in.str(all.str());
    }
    std::string next(const std::string& what) {
        std::string w;
        if (!(in >> w)) throw Fail("unexpected end of file while reading " + what);
        return w;
    }
    void skip() { next("a label"); }
    double num(const std::string& what) {
        double v;
        if (!(in >> v)) {
            in.clear();
            std::string w;
            in >> w;
            throw Fail("not a number for " + what + ": " + (w.empty() ? "end of file" : w));
        }
        return v;
    }
    // a value the reference reads as a word and converts with std::stod (the species' constants
    // and the values in zones, phaseInitialization.cpp:272-279,357-359)
    double word(const std::string& what) {
        const std::string w = next(what);
        try {
            return std::stod(w);
        } catch (...) {
            throw Fail("not a number for " + what + ": " + w);
        }
    }
};

// onOffMap of globalConstants.hpp
inline bool onOff(const std::string& s, const std::string& what) {
    if (s == "on" || s == "yes") return true;
    if (s == "off" || s == "no") return false;
    throw Fail("Unknown " + what + " flag.");
}

// ---------------------------------------------------------------- zones of the initial fields
// zone.cpp:25-125 and its shapes (src/service/zoneUnderPlane(s).cpp, zoneInsideSphere.cpp,
// zoneInsideCylinder.cpp, outerZone.cpp) on the geometry of src/primitives/plane.cpp,
// sphere.cpp, cylinder.cpp and line.cpp: a cell takes the values of the first zone that holds
// its centre.  Vector arithmetic as the reference's (component-wise, dot products summed from
// the first component, magnitudes by the 3-argument std::hypot).
struct Vec3 {
    double x[3];
};
inline Vec3 vsub(const Vec3& a, const Vec3& b) { return {{a.x[0] - b.x[0], a.x[1] - b.x[1], a.x[2] - b.x[2]}}; }
inline Vec3 vscale(double s, const Vec3& a) { return {{s * a.x[0], s * a.x[1], s * a.x[2]}}; }
inline Vec3 vdivs(const Vec3& a, double s) { return {{a.x[0] / s, a.x[1] / s, a.x[2] / s}}; }
inline double vdot(const Vec3& a, const Vec3& b) {
    double r = 0;
    for (int i = 0; i < 3; ++i) r += a.x[i] * b.x[i];
    return r;
}
inline double vmag(const Vec3& a) { return std::hypot(a.x[0], a.x[1], a.x[2]); }

struct ZonePlane {  // plane(n, p): normale n / |n|
    Vec3 n, p;
    ZonePlane(const Vec3& nn, const Vec3& pp) : n(vdivs(nn, vmag(nn))), p(pp) {}
    bool under(const Vec3& q) const { return vdot(vsub(p, q), n) >= 0; }
};

struct Zone {
    enum Kind { PLANES, SPHERE, CYLINDER, OUTER } kind = OUTER;
    std::vector<ZonePlane> planes;  // PLANES (one for "plane"), the two caps of CYLINDER
    Vec3 c{};                       // SPHERE centre, CYLINDER axis point
    Vec3 t{};                       // CYLINDER axis tangent
    double r = 0;
    bool contains(const Vec3& q) const {
        switch (kind) {
        case PLANES: {
            bool in = true;
            for (const ZonePlane& pl : planes) in = in && pl.under(q);
            return in;
        }
        case SPHERE: return vmag(vsub(q, c)) <= r;
        case CYLINDER: {
            bool in = true;
            for (const ZonePlane& pl : planes) in = in && pl.under(q);
            const Vec3 w = vsub(c, q);
            return in && vmag(vsub(w, vscale(vdot(w, t), t))) <= r;
        }
        default: return true;
        }
    }
};

inline std::vector<Zone> readZones(const std::string& path) {
    Tokens t(path);
    t.skip();
    const long long nz = (long long)t.num("number of zones");
    t.skip();
    bool outer;
    try {
        outer = onOff(t.next("outer zone flag"), "outer zone");
    } catch (const Fail&) {
        throw Fail("Unknown flag for outer zone description.");
    }
    t.skip();
    auto vec = [&](const char* what) {
        Vec3 v;
        for (double& x : v.x) x = t.num(what);
        return v;
    };
    auto radius = [&]() {
        const double r = t.num("zone radius");
        if (r <= 0) throw Fail("Radius cannot be less or equal zero.");
        return r;
    };
    std::vector<Zone> zones;
    for (long long z = 0; z < nz; ++z) {
        const std::string type = t.next("zone type");
        Zone zn;
        if (type == "plane" || type == "planes") {
            zn.kind = Zone::PLANES;
            const long long np = type == "plane" ? 1 : (long long)t.num("number of planes");
            for (long long q = 0; q < np; ++q) {
                const Vec3 n = vec("plane normal");
                t.skip();
                zn.planes.emplace_back(n, vec("plane point"));
            }
        } else if (type == "sphere") {
            zn.kind = Zone::SPHERE;
            zn.c = vec("sphere centre");
            zn.r = radius();
        } else if (type == "cylinder") {
            zn.kind = Zone::CYLINDER;
            const Vec3 n1 = vec("cylinder axis");
            t.skip();
            const Vec3 c1 = vec("cylinder base point");
            t.skip();
            const Vec3 c2 = vec("cylinder top point");
            const double r = radius();
            // cylinder.cpp: caps plane(n1 / |n1|, c1), plane(-n1 / |-n1|, c2) (each plane divides by
            // the length again), axis line(n1 / |n1|, c2)
            const Vec3 u = vdivs(n1, vmag(n1));
            const Vec3 n2 = vscale(-1, n1);
            zn.planes.emplace_back(u, c1);
            zn.planes.emplace_back(vdivs(n2, vmag(n2)), c2);
            zn.t = vdivs(u, vmag(u));
            zn.c = c2;
            zn.r = r;
        } else {
            throw Fail("Unknown zone type.");
        }
        zones.push_back(zn);
    }
    if (outer) zones.push_back(Zone{});
    return zones;
}

inline int bcType(const std::string& s) {
    if (s == "blank") return 0;  // patches of unused axes
    if (s == "freeBoundary") return FV_BC_FREE;
    if (s == "slip") return FV_BC_SLIP;
    if (s == "fixedValueCell") return FV_BC_FIXED_CELL;
    if (s == "fixedValueSurface") return FV_BC_FIXED_SURFACE;
    // boundaryConditionFromString.cpp:12-32
    if (s == "innerSurface") throw Fail("<<innerSurface>> can not be boundary surface type.");
    if (s == "subPatches") throw Fail("subPatches: patches split into sub-patches are not part of this step");
    throw Fail("Unknown type of boundary condition");
}

inline int limiterIndex(const std::string& s) {
    static const char* names[] = {"zero",       "minmod",  "vanLeer", "linear", "vanAlbada",
                                  "HQUICK",     "vanLeer2", "superbee", "vanAlbada2", "minmod2",
                                  "Sweby",      "Koren",   "Koren2",  "UTCDFS", "Schmidtmann"};
    for (int i = 0; i < 15; ++i)
        if (s == names[i]) return i;
    throw Fail("unknown TVD limiter " + s);
}

struct Deck {
    std::string dir;
    fv_config cfg{};
    double tEnd = 0;
    long long freq = 1;
    double minTime = 0;
    std::string units, eos, readFrom;
    std::vector<Zone> zones;                  // zones of the initial fields, the outer one last
    std::vector<std::vector<double>> zoneC;   // [k][zone] concentration c_k
    std::vector<double> zoneV, zoneP;         // [3 * zone + q] velocity, [zone] pressure
    bool width1D = false;                     // 1D task with #Calculation_of_mixing_zone_width on
    double hPlanck = 0;

    std::string path(const std::string& rel) const { return dir + "/" + rel; }
};

// sub_k / velocity / pressure: six patch conditions, then the values of every zone.  Only
// fixedValueCell carries values in the deck (phaseInitialization.cpp:290-299,477-487); they are
// stream extractions, and when one is not a number the reference's stream fails, the next
// patch's condition reads as empty ("Unknown type of boundary condition") or, after the last
// patch, the values label is missed ("Wrong position in file.").
inline void readPatches(Tokens& t, int nval, int field, int k, fv_config& c) {
    for (int patch = 0; patch < 6; ++patch) {
        t.skip();  // #<Patch>_boundary_condition
        const std::string type = t.next("boundary condition");
        const int bt = bcType(type);
        double v[3] = {0, 0, 0};
        if (bt == FV_BC_FIXED_CELL)
            for (int q = 0; q < nval; ++q) {
                try {
                    v[q] = t.num("boundary value");
                } catch (const Fail&) {
                    throw Fail(patch < 5 ? "Unknown type of boundary condition" : "Wrong position in file.");
                }
            }
        if (field == 0) {
            c.bc_conc[patch][k] = bt;
            c.bc_conc_value[patch][k] = v[0];
        } else if (field == 1) {
            c.bc_vel[patch] = bt;
            for (int q = 0; q < 3; ++q) c.bc_vel_value[patch][q] = v[q];
        } else {
            c.bc_p[patch] = bt;
            c.bc_p_value[patch] = v[0];
        }
    }
}

inline Deck readDeck(const std::string& dir, bool createResult) {
    Deck d;
    d.dir = dir;
    fv_config& c = d.cfg;
    // g.txt
    {
        Tokens t(d.path("set/g.txt"));
        t.skip();
        const std::string on = t.next("gravity flag");
        t.skip();
        for (int q = 0; q < 3; ++q) c.g[q] = t.num("g");
        t.skip();
        for (int q = 0; q < 3; ++q) c.g_delta[q] = t.num("g growth");
        c.gravity = onOff(on, "gravitation");
    }
    // main.txt
    std::string limiter, diffusion, turbulence, flux, dims, sourceTime, reconstruction, order, width, sle;
    {
        Tokens t(d.path("set/main.txt"));
        t.skip();
        for (int q = 0; q < 3; ++q) c.L[q] = t.num("system size");
        t.skip();
        for (int q = 0; q < 3; ++q) c.n[q] = (int)t.num("number of cells");
        t.skip(); d.tEnd = t.num("time of calculation");
        t.skip(); c.courant = t.num("Courant number");
        t.skip(); d.freq = (long long)t.num("frequency of output");
        t.skip(); d.minTime = t.num("minimal time step");
        t.skip(); c.n_species = (int)t.num("number of components");
        t.skip(); d.units = t.next("gas constant");
        t.skip(); d.eos = t.next("equation of state");
        t.skip(); limiter = t.next("limiter");
        t.skip(); c.sle_max_iter = (int)t.num("iterations");
        t.skip(); diffusion = t.next("diffusion flag");
        t.skip(); turbulence = t.next("turbulence flag");
        t.skip(); sle = t.next("matrix solver");
        t.skip(); t.next("source type");
        t.skip(); flux = t.next("flow solver");
        t.skip(); dims = t.next("dimensions");
        t.skip(); c.const_timestep = t.num("constant time step");
        t.skip(); sourceTime = t.next("source time step flag");
        t.skip(); reconstruction = t.next("reconstruction");
        t.skip(); order = t.next("approximation order");
        t.skip(); d.readFrom = t.next("start point");
        t.skip(); width = t.next("mixing zone width flag");
        // #Nonlinearity_iterations (Schemi.cpp:304, on / off): without turbulence the stage's
        // non-linearity loop ends after its first pass either way (its measure is the change of
        // epsilon, 0)
        t.skip(); onOff(t.next("nonlinearity iterations"), "nonlinearity iterations");
    }
    c.diffusion = onOff(diffusion, "diffusion");
    if (onOff(turbulence, "turbulence"))
        throw Fail("#Turbulence_flag on: turbulence models are not part of this step");
    if (reconstruction != "linear" && reconstruction != "star") throw Fail("Unknown reconstruction flag.");
    c.linear_reconstruction = reconstruction == "linear";
    // abstractMatrixSolver.cpp:51-70
    if (sle == "explicit") c.sle_solver = FV_SLE_EXPLICIT;
    else if (sle == "noSolver") c.sle_solver = FV_SLE_NO_SOLVER;
    else if (sle == "GaussSeidel") c.sle_solver = FV_SLE_GAUSS_SEIDEL;
    else if (sle == "Jacobi") c.sle_solver = FV_SLE_JACOBI;
    else if (sle == "Thomas" && dims == "1D") c.sle_solver = FV_SLE_THOMAS;
    else if (sle == "conjugateGradient") c.sle_solver = FV_SLE_CG;
    else if (sle == "JacobiConjugateGradient") c.sle_solver = FV_SLE_JACOBI_CG;
    else if (sle == "biConjugateGradient") c.sle_solver = FV_SLE_BICG;
    else throw Fail("Unknown or inappropriate matrix solver flag.");
    // "Gpu" + an order name: the factory string under which the step-solver adapter runs the
    // step inside the reference's main (schemi_adapter/gpuStepSolver.hpp)
    if (order.rfind("Gpu", 0) == 0) order = order.substr(3);
    if (order == "SecondOrder") c.order = FV_ORDER_SECOND;
    else if (order == "SecondOrderRK") c.order = FV_ORDER_SECOND_RK;
    else if (order == "ThirdOrder") c.order = FV_ORDER_THIRD;
    else if (order == "ThirdOrderCada") c.order = FV_ORDER_THIRD_CADA;
    else throw Fail("Unknown gas dynamics approximation order.");  // abstractStepSolver.cpp:87-94
    d.width1D = onOff(width, "mixed zone width calculation") && dims == "1D";
    c.dims = dims == "1D" ? 1 : dims == "2D" ? 2 : dims == "3D" ? 3 : 0;
    if (!c.dims) throw Fail("unknown #Dimensions_of_the_task " + dims);
    for (int q = c.dims; q < 3; ++q) c.n[q] = 1;
    c.limiter = limiterIndex(limiter);
    if (flux == "HLLC") c.flux = FV_FLUX_HLLC;
    else if (flux == "HLL") c.flux = FV_FLUX_HLL;
    else throw Fail("#Type_of_flow_solver " + flux + ": HLLC and HLL are implemented");
    // abstractMixtureThermodynamics.cpp:39-51
    if (d.eos == "ideal") c.eos = FV_EOS_IDEAL;
    else if (d.eos == "vanDerWaals") c.eos = FV_EOS_VAN_DER_WAALS;
    else if (d.eos == "RedlichKwong") c.eos = FV_EOS_REDLICH_KWONG;
    else if (d.eos == "stiffened") c.eos = FV_EOS_STIFFENED;
    else if (d.eos == "Kataoka") c.eos = FV_EOS_KATAOKA;
    else throw Fail("Unknown type of equation of state.");
    // phaseInitialization.cpp:418-435
    if (d.units == "SI") { c.R = kRSI; d.hPlanck = kPlanckSI; }
    else if (d.units == "1") { c.R = 1; d.hPlanck = kPlanckSI / kRSI; }
    else if (d.units == "CGS") { c.R = kRSI * 1E7; d.hPlanck = kPlanckSI * 1E7; }
    else if (d.units == "CGmS") { c.R = kRSI * 1E1; d.hPlanck = kPlanckSI * 1E4; }
    else throw Fail("Unknown type of universal gas constant.");
    c.min_timestep = d.minTime;
    // "<type>=<source coefficient>,<diffusion coefficient>" (Schemi.cpp:180-243)
    {
        const size_t eq = sourceTime.find('='), com = sourceTime.find(',');
        const auto count = [&](char ch) { return std::count(sourceTime.begin(), sourceTime.end(), ch); };
        if ((count('=') != 1 && count(',') != 1) || eq > com)
            throw Fail("Wrong format of time-step parameters settings");
        const std::string type = sourceTime.substr(0, eq == std::string::npos ? 0 : eq);
        // the two coefficients: between '=' and ',', and after ',' (std::stod, Schemi.cpp:219-226)
        const auto coeff = [&](const std::string& txt) {
            try {
                return std::stod(txt);
            } catch (const std::exception&) {
                throw Fail("Wrong format of time-step parameters settings");
            }
        };
        c.dt_coeff_source = coeff(sourceTime.substr(eq + 1, com - eq - 1));
        c.dt_coeff_diffusion = coeff(sourceTime.substr(com + 1));
        if (type != "Courant" && type != "Courant-Source" && type != "Courant-Source-Diffusion")
            throw Fail("Unknown source time-step flag.");
        c.courant_only = type == "Courant";
        c.diffusion_timestep = type == "Courant-Source-Diffusion";
    }
    c.precision = FV_PREC_F64;
    if (c.n_species < 1 || c.n_species > FV_MAX_SPECIES) throw Fail("number of components must be 1..4");
    // Schemi.cpp:312-330: a fresh run recreates result/Time.tsv once main.txt is read, before the
    // zones and the species' files (so a deck refused there still leaves it behind)
    if (createResult && (d.readFrom == "no" || d.readFrom == "initialisation")) {
        std::filesystem::create_directories(d.path("result"));
        std::ofstream(d.path("result/Time.tsv")).close();
    }
    d.zones = readZones(d.path("set/zonesDescription.txt"));
    if (c.diffusion) {
        // phaseInitialization.cpp:193-243: model, mu, D, kappa, enthalpy-flow flag, molar-mass flag
        if (!std::filesystem::exists(d.path("set/transportCoefficients.txt")))
            throw Fail("./set/transportCoefficients.txt not found.");
        Tokens t(d.path("set/transportCoefficients.txt"));
        t.skip(); const std::string model = t.next("transport model");
        t.skip(); c.mu_const = t.num("viscosity coefficient");
        t.skip(); c.D_const = t.num("diffusion coefficient");
        t.skip(); c.kappa_const = t.num("heat conduction coefficient");
        t.skip(); const std::string enthalpy = t.next("enthalpy flow flag");
        t.skip(); const std::string molMass = t.next("molar mass diffusion flag");
        if (model == "constant") c.transport = FV_TRANSPORT_CONSTANT;
        else if (model == "hardSpheres") c.transport = FV_TRANSPORT_HARD_SPHERES;
        else if (model == "LennardJones") c.transport = FV_TRANSPORT_LENNARD_JONES;
        else throw Fail("Unknown flag for transport model.");
        if (enthalpy == "no") c.enthalpy_flow = FV_ENTHALPY_NO;
        else if (enthalpy == "explicit") c.enthalpy_flow = FV_ENTHALPY_EXPLICIT;
        else if (enthalpy == "implicit") c.enthalpy_flow = FV_ENTHALPY_IMPLICIT;
        else throw Fail("Unknown flag for enthalpy flow calculation.");
        if (molMass != "on" && molMass != "off" && molMass != "yes" && molMass != "no")
            throw Fail("Unknown flag for molar mass diffusion correction.");
        c.molmass_diffusion = onOff(molMass, "molar mass diffusion correction");
        if (c.order != FV_ORDER_SECOND) throw Fail("#Diffusion_flag on: the diffusion stage runs with SecondOrder");
        if (c.flux != FV_FLUX_HLLC) throw Fail("#Diffusion_flag on: the diffusion stage runs with HLLC");
        if (c.eos != FV_EOS_IDEAL && c.eos != FV_EOS_VAN_DER_WAALS)
            throw Fail("#Diffusion_flag on: the diffusion stage runs with ideal and vanDerWaals mixtures");
    }
    const size_t nzv = d.zones.size();
    for (int k = 0; k < c.n_species; ++k) {
        Tokens t(d.path("set/sub_" + std::to_string(k + 1) + ".txt"));
        t.skip(); c.M[k] = t.word("molar mass");
        t.skip(); c.Cv[k] = t.word("Cv");
        t.skip(); c.Tc[k] = t.word("Tc");
        t.skip(); c.Pc[k] = t.word("Pc");
        // #Kinetic_diameter_(A), #Lennard_Jones_eps/kB_(K), #Lennard_Jones_sigma_(A): the
        // species data of the transport models, converted (std::stod) only by the model that
        // reads them (abstractTransportModel.cpp:44-75)
        std::string tr[3];
        for (int q = 0; q < 3; ++q) { t.skip(); tr[q] = t.next("transport parameter"); }
        auto conv = [&](const std::string& w, const char* what) {
            try {
                return std::stod(w);
            } catch (...) {
                throw Fail(std::string("not a number for ") + what + ": " + w);
            }
        };
        if (c.diffusion && c.transport == FV_TRANSPORT_HARD_SPHERES)
            c.transport_diameter[k] = conv(tr[0], "kinetic diameter");
        if (c.diffusion && c.transport == FV_TRANSPORT_LENNARD_JONES) {
            c.transport_lj_eps[k] = conv(tr[1], "Lennard-Jones eps/kB");
            c.transport_lj_sigma[k] = conv(tr[2], "Lennard-Jones sigma");
        }
        readPatches(t, 1, 0, k, c);
        if (t.next("values label") != "#Values_in_zones") throw Fail("Wrong position in file.");
        d.zoneC.emplace_back();
        for (size_t z = 0; z < nzv; ++z) d.zoneC[k].push_back(t.word("zone concentration"));
    }
    // the EOS data files of createThermodynamics (abstractMixtureThermodynamics.cpp:71-143)
    if (c.eos == FV_EOS_STIFFENED) {
        Tokens t(d.path("set/stiffenedFluidData.txt"));
        for (int k = 0; k < c.n_species; ++k) {
            t.next("species label");
            c.stiff_p0[k] = t.num("p0");
            c.stiff_gamma[k] = t.num("gamma");
        }
    } else if (c.eos == FV_EOS_KATAOKA) {
        Tokens t(d.path("set/KataokaVanDerWaalsFluidData.txt"));
        for (int k = 0; k < c.n_species; ++k) {
            t.next("species label");
            c.lj_eps[k] = t.num("Lennard-Jones epsilon");
            c.lj_sigma[k] = t.num("Lennard-Jones sigma");
        }
        t.skip();
        const std::string rule = t.next("b calculation");
        c.kataoka_b_coeff = t.num("b coefficient");
        if (rule == "critical") c.kataoka_b_critical = 1;
        else if (rule == "Kataoka") c.kataoka_b_critical = 0;
        else throw Fail("Wrong type of Kataoka-van der Waals b coefficient calculation");
    }
    {
        Tokens t(d.path("set/velocity.txt"));
        readPatches(t, 3, 1, 0, c);
        if (t.next("values label") != "#Values_in_zones") throw Fail("Wrong position in file.");
        for (size_t z = 0; z < 3 * nzv; ++z) d.zoneV.push_back(t.word("zone velocity"));
    }
    {
        Tokens t(d.path("set/pressure.txt"));
        readPatches(t, 1, 2, 0, c);
        if (t.next("values label") != "#Values_in_zones") throw Fail("Wrong position in file.");
        for (size_t z = 0; z < nzv; ++z) d.zoneP.push_back(t.word("zone pressure"));
    }
    // chemistry
    {
        Tokens t(d.path("set/chemicalKinetics.txt"));
        t.skip();
        const std::string name = t.next("reaction name");
        if (name == "no") {
            c.chemistry = FV_CHEM_NONE;
        } else if (name == "Cl2") {
            c.chemistry = FV_CHEM_CL2;
            double v[6];
            for (double& x : v) { t.skip(); x = t.num("Arrhenius parameter"); }
            c.chem_forward = fv_arrhenius{v[0], v[1], v[2]};
            c.chem_backward = fv_arrhenius{v[3], v[4], v[5]};
            t.skip();
            const std::string solver = t.next("chemical solver");
            static const std::map<std::string, int> solvers = {
                {"Gauss-Seidel", FV_CHEM_GAUSS_SEIDEL}, {"Jacobi", FV_CHEM_JACOBI},
                {"GaussElimination", FV_CHEM_GAUSS_ELIMINATION}, {"conjugateGradient", FV_CHEM_CONJUGATE_GRADIENT},
                {"JacobiConjugateGradient", FV_CHEM_JACOBI_CONJUGATE_GRADIENT}};
            auto it = solvers.find(solver);
            if (it == solvers.end()) throw Fail("Unknown type of chemical iterative solver.");
            c.chem_solver = it->second;
            t.skip();
            c.chem_max_iter = (int)t.num("chemical solver iterations");
        } else {
            throw Fail("chemical mechanism " + name + " is not implemented (no, Cl2)");
        }
    }
    return d;
}


}  // namespace fvdeck
