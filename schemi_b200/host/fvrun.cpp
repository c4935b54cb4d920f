// fvrun -- runs a Schemi task deck on the GPU through the C-ABI of include/fvstep.h and writes the
// reference's result files.
//
//     fvrun [deck_directory]            (default: the current directory)
//     fvrun --print-config [deck_dir]   parse the deck and print the fv_config it maps to (no GPU)
//
// The deck is what the reference reads (paths inside the Schemi project): set/main.txt (the 24
// positional keys of main/Schemi.cpp:101-163), set/g.txt (:83-99), set/sub_<k>.txt,
// set/velocity.txt, set/pressure.txt (phaseInitialization.cpp), set/chemicalKinetics.txt
// (Schemi.cpp:672-716, chemicalKineticsChlorumDissociation.cpp:275-308) and
// set/zonesDescription.txt (zone.cpp: planes, spheres, cylinders, the outer zone) with the
// optional set/sub_<k>_modifFunction.txt of a fresh run.  The time loop, its output schedule, the restart from
// fieldsOutput/output_<N> + result/Time.tsv and the last-step clamp follow Schemi.cpp:312-573,
// 664-670, 716-940; the files written follow output::dataOutput (src/service/output.cpp:14-308):
// result/output_<NNNNNN>.tsv, result/Time.tsv, fieldsOutput/output_<NNNNNN>/*.dat and
// timeOfCalculation.tsv, with the reference's 20 significant digits.
//
// A 1D task with #Calculation_of_mixing_zone_width on also writes result/timeWidth.tsv
// (output::mixedZoneWidth1D).  Not supported (the run stops with a message): diffusion,
// turbulence, and chemical mechanisms other than "no" and "Cl2".
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "deck.hpp"
#include "fvstep.h"

namespace {
using namespace fvdeck;

// ---------------------------------------------------------------- geometry (cell centres)
// node coordinates 0 + d*i and the 8-corner average of the mesh generator (mesh.cpp:296-1900)
std::vector<double> centres(const fv_config& c, int a) {
    const bool used = a < c.dims;
    const int n = used ? c.n[a] : 1;
    const double L = c.L[a], d = L / n;
    auto node = [&](int i) -> double {
        if (used) return 0.0 + d * (double)(size_t)i;
        return i == 0 ? 0.0 : L;
    };
    std::vector<double> out(n);
    for (int i = 0; i < n; ++i) {
        const double A = node(i), B = node(i + 1);
        double seq[8];
        for (int q = 0; q < 8; ++q) {
            const int bit = a == 0 ? (q & 1) : (a == 1 ? ((q >> 1) & 1) : ((q >> 2) & 1));
            seq[q] = bit ? B : A;
        }
        double s = seq[0] + seq[1];
        for (int q = 2; q < 8; ++q) s = s + seq[q];
        out[i] = s / 8.;
    }
    return out;
}

// Initial fields of a fresh run (phaseInitialization.cpp:1160-1310): every cell takes the values
// of the first zone holding its centre, then a species' concentration is scaled by the optional
// set/sub_<k>_modifFunction.txt ("gaussian": A + B exp(-((x - x0) / c)^2) of the centre's x).
void initialFields(const Deck& d, const fv_config& c, std::vector<std::vector<double>>& prim) {
    const int N = c.n_species;
    const std::vector<double> cx = centres(c, 0), cy = centres(c, 1), cz = centres(c, 2);
    const long long nc = (long long)c.n[0] * c.n[1] * c.n[2];
    auto zoneOf = [&](long long i, const std::string& what) -> size_t {
        const long long ix = i % c.n[0], iy = (i / c.n[0]) % c.n[1], iz = i / ((long long)c.n[0] * c.n[1]);
        const Vec3 rc{{cx[ix], cy[iy], cz[iz]}};
        for (size_t z = 0; z < d.zones.size(); ++z)
            if (d.zones[z].contains(rc)) return z;
        throw Fail("Cell " + std::to_string(i) + " of " + what + " dropped out of all zones.");
    };
    for (int k = 0; k < N; ++k) {
        for (long long i = 0; i < nc; ++i)
            prim[k][i] = d.zoneC[k][zoneOf(i, std::to_string(k + 1) + " component concentration")];
        std::ifstream mf(d.path("set/sub_" + std::to_string(k + 1) + "_modifFunction.txt"));
        if (!mf.is_open()) continue;
        std::string skip, name;
        mf >> skip >> name;
        if (name != "gaussian") continue;  // other names leave the field as it is
        double A, B, x0, w;
        mf >> skip >> A >> skip >> B >> skip >> x0 >> skip >> w;
        for (long long i = 0; i < nc; ++i) {
            const double u = (cx[i % c.n[0]] - x0) / w;
            prim[k][i] *= A + B * std::exp(-(u * u));
        }
    }
    for (long long i = 0; i < nc; ++i) {
        const size_t z = zoneOf(i, "velocity");
        for (int q = 0; q < 3; ++q) prim[N + q][i] = d.zoneV[3 * z + q];
    }
    for (long long i = 0; i < nc; ++i) prim[N + 3][i] = d.zoneP[zoneOf(i, "pressure")];
}

// ---------------------------------------------------------------- Helmholtz energy and entropy
// mixtureIdeal::Fv/Sv (mixtureIdeal.cpp:300-354), mixtureVanDerWaals::Fv/Sv (:461-537) with
// idealFluid::Fmx/Smx (idealFluid.cpp:90-116) and vanDerWaalsFluid::Fmx/Smx (:122-151).
// With the mixtures of mixtureRedlichKwong::Fv/Sv (:459-530, RedlichKwongFluid::Fmx/Smx :175-211),
// mixtureStiffened::Fv/Sv (:390-470, stiffenedFluid::Fmx/Smx :91-120) and
// mixtureKataokaVanDerWaals::Fv/Sv (KataokaVanDerWaalsFluid::Fmx/Smx :430-496).
struct Thermo {
    int N, eos;
    double R, kB, h;
    double molecMass[FV_MAX_SPECIES];
    // per molecule: van der Waals / Redlich-Kwong a and b, Kataoka V0, eps and b; stiffened p0
    double aMolec[FV_MAX_SPECIES][FV_MAX_SPECIES] = {}, bMolec[FV_MAX_SPECIES][FV_MAX_SPECIES] = {};
    double V0Molec[FV_MAX_SPECIES][FV_MAX_SPECIES] = {}, epsMolec[FV_MAX_SPECIES][FV_MAX_SPECIES] = {};
    double p0[FV_MAX_SPECIES][FV_MAX_SPECIES] = {};

    Thermo(const fv_config& c, double hPlanck) : N(c.n_species), eos(c.eos), R(c.R), kB(c.R / kNA), h(hPlanck) {
        double a[FV_MAX_SPECIES][FV_MAX_SPECIES] = {}, b[FV_MAX_SPECIES][FV_MAX_SPECIES] = {};
        double V0[FV_MAX_SPECIES][FV_MAX_SPECIES] = {}, ep[FV_MAX_SPECIES][FV_MAX_SPECIES] = {};
        constexpr double chi{std::cbrt(2) - 1.};  // mixtureRedlichKwong.cpp:34-37
        constexpr double Sigma_a{1. / (9. * chi)}, Sigma_b{chi / 3.};
        for (int k = 0; k < N; ++k) {
            molecMass[k] = c.M[k] / kNA;
            if (eos == FV_EOS_REDLICH_KWONG) {
                b[k][k] = Sigma_b * R * c.Tc[k] / c.Pc[k];
                a[k][k] = Sigma_a * R * R * c.Tc[k] * c.Tc[k] * std::sqrt(c.Tc[k]) / c.Pc[k];
            } else if (eos == FV_EOS_KATAOKA) {
                const double sg = c.lj_sigma[k];
                b[k][k] = c.kataoka_b_critical ? c.kataoka_b_coeff * R * c.Tc[k] / (8 * c.Pc[k])
                                               : c.kataoka_b_coeff * (sg * sg * sg) * kNA;
                V0[k][k] = (sg * sg * sg) / std::sqrt(2) * kNA;
                ep[k][k] = c.lj_eps[k];
            } else {
                b[k][k] = c.Tc[k] * R / (8 * c.Pc[k]);
                a[k][k] = c.Pc[k] * b[k][k] * b[k][k] * 27;
            }
            p0[k][k] = c.stiff_p0[k];
        }
        for (int k = 0; k < N; ++k)
            for (int l = 0; l < N; ++l)
                if (k != l) {
                    b[k][l] = std::pow(0.5 * (std::cbrt(b[k][k]) + std::cbrt(b[l][l])), 3);
                    a[k][l] = std::sqrt(a[k][k] * a[l][l]);
                    V0[k][l] = std::pow(0.5 * (std::cbrt(V0[k][k]) + std::cbrt(V0[l][l])), 3);
                    ep[k][l] = std::sqrt(ep[k][k] * ep[l][l]);
                    p0[k][l] = std::sqrt(p0[k][k] * p0[l][l]);
                }
        for (int k = 0; k < N; ++k)
            for (int l = 0; l < N; ++l) {
                bMolec[k][l] = b[k][l] / kNA;
                aMolec[k][l] = a[k][l] / (kNA * kNA);
                V0Molec[k][l] = V0[k][l] / kNA;
                epsMolec[k][l] = ep[k][l] / kNA;
            }
    }

    // KataokaVanDerWaalsFluid::qa with the molecular constants (M = 13 terms)
    static double qa(double c, double T, double V0, double eps, double R) {
        const double V0c{V0 * c};
        const double epsRT{0.5 * eps / (R * T)};
        double series{1.0};
        for (std::size_t J = 2; J <= 13; ++J) series += std::pow(V0c, (J - 1.) / 3.) * std::exp((J - 1.) * epsRT);
        return series;
    }

    // Sum over the species of a valarray expression, in the order libstdc++'s _Expr::sum() takes:
    // from the last element down to the first.
    template <class Term>
    double speciesSum(Term term) const {
        double s = term(N - 1);
        for (int k = N - 2; k >= 0; --k) s += term(k);
        return s;
    }

    // F (first) and S (second) per volume of a cell
    void FS(const double* c, double T, double& F, double& S) const {
        double x[FV_MAX_SPECIES] = {}, lam3[FV_MAX_SPECIES] = {};
        for (int k = 0; k < N; ++k) x[k] = c[k + 1] / c[0];
        const double molecConc = c[0] * kNA;
        const double Vm = 1 / molecConc;
        for (int k = 0; k < N; ++k) {
            const double lam = std::sqrt((h * h) / (2 * kPi * molecMass[k] * kB * T));
            lam3[k] = lam * lam * lam;
        }
        const double A = speciesSum([&](int k) { return x[k] * std::log(x[k] + kStab); });
        const double C = speciesSum([&](int k) { return -x[k] * std::log(x[k] + kStab); });
        if (eos == FV_EOS_IDEAL || eos == FV_EOS_STIFFENED) {
            const double B = speciesSum([&](int k) { return x[k] * std::log(Vm / lam3[k]); });
            if (eos == FV_EOS_IDEAL) {
                F = kB * T * (A - 1 - B) * molecConc;
            } else {
                double p0m = 0;
                for (int k = 0; k < N; ++k)
                    for (int l = 0; l < N; ++l) p0m += x[k] * x[l] * p0[k][l];
                F = (kB * T * (A - 1 - B) + p0m * Vm) * molecConc;
            }
            S = kB * (C + B + 5. / 2.) * molecConc;
            return;
        }
        if (eos == FV_EOS_REDLICH_KWONG || eos == FV_EOS_KATAOKA) {
            double am = 0, bm = 0, V0m = 0, em = 0;
            for (int k = 0; k < N; ++k)
                for (int l = 0; l < N; ++l) {
                    if (eos == FV_EOS_KATAOKA) {
                        V0m += x[k] * x[l] * V0Molec[k][l];
                        em += x[k] * x[l] * epsMolec[k][l];
                    } else {
                        am += x[k] * x[l] * aMolec[k][l];
                    }
                    bm += x[k] * x[l] * bMolec[k][l];
                }
            const double mixS = -A;
            const double trans = speciesSum([&](int k) { return x[k] * std::log((Vm - bm) / lam3[k]); });
            if (eos == FV_EOS_REDLICH_KWONG) {
                const double potF = am / (bm * std::sqrt(T)) * std::log1p(bm / Vm);
                const double potS = 0.5 * am / (bm * T * std::sqrt(T)) * std::log1p(bm / Vm);
                F = (kB * T * (A - 1 - trans) - potF) * molecConc;
                S = (kB * (mixS + 5. / 2. + trans) - potS) * molecConc;
                return;
            }
            const double q = qa(1 / Vm, T, V0m, em, kB);
            const double potF = std::log(q);
            const double V0c{V0m / Vm};
            const double epsRT{0.5 * em / (kB * T)};
            double series{0.0};
            for (std::size_t J = 2; J <= 13; ++J)
                series -= 0.5 * (J - 1) * std::pow(V0c, (J - 1) / 3.) * std::exp(0.5 * (J - 1.) * epsRT);
            const double potS = std::log(q) + em / (kB * T) * series / q;
            F = kB * T * ((A - 1 - trans) - potF) * molecConc;
            S = kB * ((mixS + 5. / 2. + trans) - potS) * molecConc;
            return;
        }
        // mixture a and b accumulate cell by cell from zero, k outer, l inner
        double am = 0, bm = 0;
        for (int k = 0; k < N; ++k)
            for (int l = 0; l < N; ++l) {
                am += x[k] * x[l] * aMolec[k][l];
                bm += x[k] * x[l] * bMolec[k][l];
            }
        const double B = speciesSum([&](int k) { return x[k] * std::log((Vm - bm) / lam3[k]); });
        F = (kB * T * (A - 1 - B) - am / Vm) * molecConc;
        // mixtureVanDerWaals::Sv divides the molecular b by Avogadro's number once more
        const double bs = bm / kNA;
        const double B2 = speciesSum([&](int k) { return x[k] * std::log((Vm - bs) / lam3[k]); });
        S = kB * (C + 5. / 2. + B2) * molecConc;
    }
};

// ---------------------------------------------------------------- output (output.cpp:14-308)
std::string number(long long n) {
    const std::string s = std::to_string(n);
    if ((int)s.size() > kNumberLength) throw Fail("Output number length larger than specified number of digits.", 3);
    return std::string(kNumberLength - s.size(), '0') + s;
}

// `sonic`, when not empty, replaces the downloaded sonic speeds: with #Constant_timestep main never
// recomputes its sonic-speed field after initialisation (Schemi.cpp:641-646, 807-812), and every
// output carries the initial values.
void writeOutput(const Deck& d, fv_handle* h, long long nOutput, double time, const Thermo& th,
                 const std::vector<double>& sonic) {
    const fv_config& c = d.cfg;
    const int N = c.n_species;
    const long long nc = (long long)c.n[0] * c.n[1] * c.n[2];
    std::vector<std::vector<double>> f(FV_F_COUNT, std::vector<double>(nc));
    std::vector<double*> ptr(FV_F_COUNT);
    for (int i = 0; i < FV_F_COUNT; ++i) ptr[i] = f[i].data();
    const fv_status st = fv_download(h, ptr.data());
    if (st != FV_OK) throw Fail(std::string("fv_download: ") + fv_last_error(h), st);
    const std::vector<double> cx = centres(c, 0), cy = centres(c, 1), cz = centres(c, 2);

    const std::string num = number(nOutput);
    std::filesystem::create_directories(d.path("result"));
    std::ofstream out(d.path("result/output_" + num + ".tsv"));
    if (!out.is_open()) throw Fail("Couldn't create outputFile.", FV_ERR_SYSTEM);
    out.precision(kPrecision);
    out << "coordinate_x" << '\t' << "coordinate_y" << '\t' << "coordinate_z" << '\t';
    for (int k = 1; k <= N; ++k) out << "concentration_" << k << '\t';
    out << "concentration" << '\t';
    for (int k = 1; k <= N; ++k) out << "x_" << k << '\t';
    for (int k = 1; k <= N; ++k) out << "density_" << k << '\t';
    out << "density" << '\t';
    for (int k = 1; k <= N; ++k) out << "w_" << k << '\t';
    out << "velocity_x\tvelocity_y\tvelocity_z\tpressure\ttemperature\tk\tepsilon\ta_x\ta_y\ta_z\tb\t"
           "turbulent_viscosity\tmomentum_x\tmomentum_y\tmomentum_z\ttotal_energy\tinternal_energy\t"
           "Helmholtz_energy\tentropy\tsonic_speed\n";
    for (long long i = 0; i < nc; ++i) {
        const long long ix = i % c.n[0], iy = (i / c.n[0]) % c.n[1], iz = i / ((long long)c.n[0] * c.n[1]);
        double cc[FV_MAX_SPECIES + 1];
        cc[0] = f[FV_F_CONC0][i];  // the state's total (an averaged field after a multi-stage step)
        for (int k = 1; k <= N; ++k) cc[k] = f[FV_F_CONC + k - 1][i];
        const double T = f[FV_F_T][i];
        double F, S;
        th.FS(cc, T, F, S);
        out << cx[ix] << '\t' << cy[iy] << '\t' << cz[iz] << '\t';
        for (int k = 1; k <= N; ++k) out << cc[k] << '\t';
        out << cc[0] << '\t';
        for (int k = 1; k <= N; ++k) out << cc[k] / cc[0] << '\t';
        for (int k = 0; k < N; ++k) out << f[FV_F_RHO_K + k][i] << '\t';
        const double rho = f[FV_F_RHO][i];
        out << rho << '\t';
        for (int k = 0; k < N; ++k) out << f[FV_F_RHO_K + k][i] / rho << '\t';
        out << f[FV_F_VX][i] << '\t' << f[FV_F_VY][i] << '\t' << f[FV_F_VZ][i] << '\t';
        out << f[FV_F_P][i] << '\t' << T << '\t';
        out << 0. << '\t' << 0. << '\t' << 0. << '\t' << 0. << '\t' << 0. << '\t' << 0. << '\t' << 0. << '\t';
        out << f[FV_F_MX][i] << '\t' << f[FV_F_MY][i] << '\t' << f[FV_F_MZ][i] << '\t';
        out << f[FV_F_E][i] << '\t' << f[FV_F_UV][i] << '\t' << F << '\t' << S << '\t'
            << (sonic.empty() ? f[FV_F_SONIC][i] : sonic[i]) << '\n';
    }
    out.close();
    {
        std::ofstream tf(d.path("result/Time.tsv"), std::ios::app);
        if (!tf.is_open()) throw Fail("Couldn't open ./result/Time.tsv.", FV_ERR_SYSTEM);
        tf.precision(kPrecision);
        tf << nOutput << '\t' << time << '\n';
    }
    // restart data (fieldsOutput/output_N): turbulence fields are zero without a turbulence model
    const std::string dir = d.path("fieldsOutput/output_" + num + "/");
    std::filesystem::create_directories(dir);
    auto file = [&](const std::string& name) {
        std::ofstream o(dir + name);
        if (!o.is_open()) throw Fail("Couldn't create output file for field data " + dir + name, FV_ERR_SYSTEM);
        o.precision(kPrecision);
        return o;
    };
    {
        auto o = file("a.dat");
        for (long long i = 0; i < nc; ++i) o << 0. << '\t' << 0. << '\t' << 0. << '\n';
    }
    for (const char* name : {"b.dat", "epsilon.dat", "k.dat"}) {
        auto o = file(name);
        for (long long i = 0; i < nc; ++i) o << 0. << '\n';
    }
    {
        auto o = file("pressure.dat");
        for (long long i = 0; i < nc; ++i) o << f[FV_F_P][i] << '\n';
    }
    {
        auto o = file("velocity.dat");
        for (long long i = 0; i < nc; ++i) o << f[FV_F_VX][i] << '\t' << f[FV_F_VY][i] << '\t' << f[FV_F_VZ][i] << '\n';
    }
    for (int k = 0; k < N; ++k) {
        auto o = file("sub_" + std::to_string(k + 1) + ".dat");
        for (long long i = 0; i < nc; ++i) o << f[FV_F_CONC + k][i] << '\n';
    }
    std::cout << "./result/output_" << num << ".tsv output file is opened. Number of output: " << nOutput << '.'
              << std::endl;
}

// restart fields of fieldsOutput/output_N (phaseInitialization.cpp:1382-1746)
std::vector<double> column(const std::string& path, long long n, int cols, int col) {
    std::ifstream f(path);
    if (!f.is_open()) throw Fail("Couldn't open " + path, FV_ERR_SYSTEM);
    std::vector<double> out(n);
    for (long long i = 0; i < n; ++i)
        for (int q = 0; q < cols; ++q) {
            double v;
            if (!(f >> v)) throw Fail("too few values in " + path);
            if (q == col) out[i] = v;
        }
    return out;
}

void printConfig(const fv_config& c, const Deck& d) {
    std::cout.precision(17);
    std::cout << "{\"dims\": " << c.dims << ", \"n\": [" << c.n[0] << ", " << c.n[1] << ", " << c.n[2] << "]"
              << ", \"L\": [" << c.L[0] << ", " << c.L[1] << ", " << c.L[2] << "]"
              << ", \"n_species\": " << c.n_species << ", \"R\": " << c.R << ", \"M\": [";
    for (int k = 0; k < c.n_species; ++k) std::cout << (k ? ", " : "") << c.M[k];
    std::cout << "], \"Cv\": [";
    for (int k = 0; k < c.n_species; ++k) std::cout << (k ? ", " : "") << c.Cv[k];
    std::cout << "], \"eos\": " << c.eos << ", \"flux\": " << c.flux << ", \"limiter\": " << c.limiter
              << ", \"courant\": " << c.courant << ", \"min_timestep\": " << c.min_timestep
              << ", \"courant_only\": " << c.courant_only << ", \"gravity\": " << c.gravity << ", \"g\": ["
              << c.g[0] << ", " << c.g[1] << ", " << c.g[2] << "], \"bc_vel\": [";
    for (int p = 0; p < 6; ++p) std::cout << (p ? ", " : "") << c.bc_vel[p];
    std::cout << "], \"bc_p\": [";
    for (int p = 0; p < 6; ++p) std::cout << (p ? ", " : "") << c.bc_p[p];
    std::cout << "], \"chemistry\": " << c.chemistry << ", \"const_timestep\": " << c.const_timestep
              << ", \"t_end\": " << d.tEnd << ", \"frequency\": " << d.freq << ", \"start\": \"" << d.readFrom
              << "\", \"order\": " << c.order << ", \"diffusion\": " << c.diffusion
              << ", \"sle_solver\": " << c.sle_solver << ", \"transport\": " << c.transport
              << ", \"mu_const\": " << c.mu_const << ", \"D_const\": " << c.D_const
              << ", \"kappa_const\": " << c.kappa_const << ", \"enthalpy_flow\": " << c.enthalpy_flow
              << ", \"molmass_diffusion\": " << c.molmass_diffusion
              << ", \"linear_reconstruction\": " << c.linear_reconstruction
              << ", \"diffusion_timestep\": " << c.diffusion_timestep
              << ", \"dt_coeff_source\": " << c.dt_coeff_source
              << ", \"dt_coeff_diffusion\": " << c.dt_coeff_diffusion << ", \"transport_diameter\": [";
    for (int k = 0; k < c.n_species; ++k) std::cout << (k ? ", " : "") << c.transport_diameter[k];
    std::cout << "], \"transport_lj_eps\": [";
    for (int k = 0; k < c.n_species; ++k) std::cout << (k ? ", " : "") << c.transport_lj_eps[k];
    std::cout << "], \"transport_lj_sigma\": [";
    for (int k = 0; k < c.n_species; ++k) std::cout << (k ? ", " : "") << c.transport_lj_sigma[k];
    std::cout << "]}" << std::endl;
}

// output::mixedZoneWidth1D (src/service/output.cpp:310-391): the distance between the first
// crossings (in cell order) of the mole fraction c_1 / c_0 through 0.01 and through 0.99, each at
// the mid-point of the two cells, or at an end of the tube when there is none; appended to
// result/timeWidth.tsv as "time<TAB>width".
void writeWidth(const Deck& d, fv_handle* h, double time) {
    const fv_config& c = d.cfg;
    const long long n = c.n[0];
    std::vector<double> c0(n), c1(n);
    std::vector<double*> ptr(FV_F_COUNT, nullptr);
    ptr[FV_F_CONC0] = c0.data();
    ptr[FV_F_CONC] = c1.data();
    const fv_status st = fv_download(h, ptr.data());
    if (st != FV_OK) throw Fail(std::string("fv_download: ") + fv_last_error(h), st);
    const std::vector<double> x = centres(c, 0);
    const double zeroMix = 0.01;
    auto X = [&](long long i) { return c1[i] / c0[i]; };
    double rL = 0, rR = 0;
    bool found = false;
    for (long long i = 0; i + 1 < n; ++i) {
        const bool b1 = X(i) >= zeroMix && X(i + 1) < zeroMix, b2 = X(i) < zeroMix && X(i + 1) >= zeroMix;
        if (b1 || b2) {
            rL = 0.5 * (x[i] + x[i + 1]);
            found = true;
            break;
        }
    }
    if (!found) rL = X(0) < X(n - 1) ? x[0] : x[n - 1];
    found = false;
    for (long long i = 0; i + 1 < n; ++i) {
        const bool b1 = X(i) > (1 - zeroMix) && X(i + 1) <= (1 - zeroMix);
        const bool b2 = X(i) <= (1 - zeroMix) && X(i + 1) > (1 - zeroMix);
        if (b1 || b2) {
            rR = 0.5 * (x[i] + x[i + 1]);
            found = true;
            break;
        }
    }
    if (!found) rR = X(0) > X(n - 1) ? x[0] : x[n - 1];
    std::ofstream f(d.path("result/timeWidth.tsv"), std::ios::app);
    if (!f.is_open()) throw Fail("Couldn't create ./result/timeWidth.tsv.", FV_ERR_SYSTEM);
    f.precision(kPrecision);
    f << time << '\t' << std::abs(rR - rL) << '\n';
}

int run(const Deck& d) {
    const fv_config& c = d.cfg;
    const int N = c.n_species;
    const long long nc = (long long)c.n[0] * c.n[1] * c.n[2];
    const Thermo th(c, d.hPlanck);
    const auto start = std::chrono::high_resolution_clock::now();
    fv_handle* h = nullptr;
    fv_status st = fv_create(&c, &h);
    if (st != FV_OK) throw Fail("fv_create failed (see the messages above)", st);
    struct Guard {
        fv_handle* h;
        ~Guard() { fv_destroy(h); }
    } guard{h};

    // restart set
    std::vector<std::vector<double>> prim(N + 4, std::vector<double>(nc));
    long long nouts = 0, nsteps = 0, noutsW = 0;
    const long long freqW = std::min(d.freq, 1000LL);  // Schemi.cpp:178
    double time = 0;
    const bool fresh = d.readFrom == "no" || d.readFrom == "initialisation";
    if (fresh) {
        initialFields(d, c, prim);
        std::filesystem::create_directories(d.path("result"));
        std::ofstream(d.path("result/Time.tsv")).close();  // recreated
        if (d.width1D) std::ofstream(d.path("result/timeWidth.tsv")) << "Time" << '\t' << "Width" << std::endl;
    } else {
        const long long point = std::stoll(d.readFrom);
        std::ifstream tf(d.path("result/Time.tsv"));
        if (!tf.is_open()) throw Fail("Couldn't open Time.tsv", FV_ERR_SYSTEM);
        std::vector<std::string> lines;
        std::string line;
        while (std::getline(tf, line)) lines.push_back(line);
        if ((long long)lines.size() <= point) throw Fail("Appropriate line wasn't found in Time.tsv", FV_ERR_SYSTEM);
        if (point == 0) throw Fail("Time.tsv contains only one line.", FV_ERR_SYSTEM);
        const std::string& ts = lines[point];
        const size_t tab = ts.find('\t');
        if (tab == std::string::npos) throw Fail("Could not find tab delimiter.");
        nouts = std::stoll(ts.substr(0, tab));
        time = std::stod(ts.substr(tab + 1));
        if (d.tEnd - time <= 0)
            throw Fail("Time of calculation lesser or equal than time of executed calculation.");
        if (nouts != point) throw Fail("Number of output does not concur with <<readDataPoint>>.", FV_ERR_SYSTEM);
        const bool last = (long long)lines.size() == point + 1;
        {
            std::ofstream nf(d.path("result/Time.tsv"));
            for (long long q = 0; q <= point; ++q) nf << lines[q] << '\n';
        }
        nsteps = nouts * d.freq;
        if (last) {
            // the step count of timeOfCalculation.tsv; 0 when the file has no "steps" word,
            // nouts * frequency when the file is missing or the count unreadable
            std::ifstream sf(d.path("timeOfCalculation.tsv"));
            if (sf.is_open()) {
                nsteps = 0;
                std::string w;
                while (sf >> w)
                    if (w == "steps") {
                        try {
                            if (!(sf >> w)) throw std::invalid_argument("no count");
                            nsteps = std::stoll(w);
                        } catch (...) {
                            nsteps = nouts * d.freq;
                        }
                        break;
                    }
            }
        }
        if (d.width1D) {
            // Schemi.cpp:478-541: the width outputs up to the restart time; the file is rewritten
            // with those lines (the header and the outputs at times not after it)
            std::vector<std::string> wlines;
            {
                std::ifstream wf(d.path("result/timeWidth.tsv"));
                if (!wf.is_open()) throw Fail("Couldn't open timeWidth.tsv", FV_ERR_SYSTEM);
                std::string wl;
                while (std::getline(wf, wl)) wlines.push_back(wl);
            }
            long long lineNumber = 0;
            for (const std::string& wl : wlines) {
                lineNumber++;
                if (lineNumber == 1) continue;
                const size_t wt = wl.find('\t');
                if (wt == std::string::npos) throw Fail("Could not find tab delimiter.");
                const double tw = std::stod(wl.substr(0, wt));
                if (tw == time) break;
                if (tw > time) {
                    lineNumber--;
                    break;
                }
            }
            noutsW = lineNumber - 1;
            std::ofstream wn(d.path("result/timeWidth.tsv"));
            if (!wn.is_open()) throw Fail("Couldn't open timeWidth.tsv", FV_ERR_SYSTEM);
            for (long long q = 0; q < lineNumber; ++q) wn << wlines[q] << '\n';
        }
        const std::string dir = d.path("fieldsOutput/output_" + number(point) + "/");
        for (int k = 0; k < N; ++k) prim[k] = column(dir + "sub_" + std::to_string(k + 1) + ".dat", nc, 1, 0);
        for (int q = 0; q < 3; ++q) prim[N + q] = column(dir + "velocity.dat", nc, 3, q);
        prim[N + 3] = column(dir + "pressure.dat", nc, 1, 0);
    }
    std::vector<const double*> pp(N + 4);
    for (int q = 0; q < N + 4; ++q) pp[q] = prim[q].data();
    if ((st = fv_upload(h, pp.data())) != FV_OK) throw Fail(std::string("fv_upload: ") + fv_last_error(h), st);
    // first step: the minimal (or constant) step, not beyond the time of calculation
    const double dt0 = std::min(c.const_timestep > 0 ? c.const_timestep : d.minTime, d.tEnd);
    if ((st = fv_set_time(h, time, dt0)) != FV_OK) throw Fail("fv_set_time", st);
    std::vector<double> sonic;
    if (c.const_timestep > 0) {
        sonic.resize(nc);
        std::vector<double*> only(FV_F_COUNT, nullptr);
        only[FV_F_SONIC] = sonic.data();
        if ((st = fv_download(h, only.data())) != FV_OK) throw Fail(std::string("fv_download: ") + fv_last_error(h), st);
    }

    if (fresh) {
        writeOutput(d, h, nouts, time, th, sonic);
        if (d.width1D) writeWidth(d, h, time);
    }
    nouts++, noutsW++;
    if (d.readFrom == "initialisation") return 0;

    while (time < d.tEnd) {
        long long next = nouts * d.freq;
        if (d.width1D) next = std::min(next, noutsW * freqW);
        const long long toGo = std::max(1LL, next - nsteps);
        fv_run_stats rs{};
        st = fv_run(h, d.tEnd, toGo, &rs);
        nsteps += rs.steps;
        time = rs.time;
        if (st != FV_OK) {
            // the failing step is the one after the last completed step; its time step is the one
            // the run would have taken next
            std::clog << fv_last_error(h) << std::endl << "Step number " << nsteps + 1 << '.' << std::endl;
            std::clog << "Time-step " << rs.dt_next << '.' << std::endl;
            std::clog << "Emergency output." << std::endl;
            writeOutput(d, h, nouts, time, th, sonic);
            return EXIT_FAILURE;  // Schemi.cpp:774-799
        }
        if (rs.steps == 0) break;
        if (nsteps == nouts * d.freq || time == d.tEnd) {
            std::cout << "Time = " << time << std::endl << "Step number = " << nsteps << std::endl;
            writeOutput(d, h, nouts, time, th, sonic);
            nouts++;
        }
        if (d.width1D && (nsteps == noutsW * freqW || time == d.tEnd)) {
            writeWidth(d, h, time);
            noutsW++;
        }
    }
    std::cout << "End" << std::endl;
    std::ofstream tc(d.path("timeOfCalculation.tsv"));
    tc.precision(kPrecision);
    tc << "Time of execution" << std::endl
       << std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::high_resolution_clock::now() - start)
              .count()
       << std::endl
       << "Number of steps" << std::endl
       << nsteps << std::endl;
    // the reference's per-stage timers; the fused kernels have no separate stages
    for (const char* stage : {"Time of TVD stage work:", "Time of Hancock stage work:", "Time of Riemann solver work:",
                              "Time of time integration work:", "Time of Diffusion solver work:"})
        tc << stage << std::endl << 0 << std::endl;
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    bool printOnly = false;
    std::string dir = ".";
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--print-config") printOnly = true;
        else if (a == "-h" || a == "--help") {
            std::cout << "usage: fvrun [--print-config] [deck_directory]" << std::endl;
            return 0;
        } else dir = a;
    }
    try {
        const Deck d = readDeck(dir, !printOnly);
        if (printOnly) {
            printConfig(d.cfg, d);
            return 0;
        }
        return run(d);
    } catch (const std::exception& e) {
        // Schemi.cpp:965-973: every error ends the run with its message and EXIT_FAILURE
        std::clog << e.what() << std::endl;
        return EXIT_FAILURE;
    }
}
