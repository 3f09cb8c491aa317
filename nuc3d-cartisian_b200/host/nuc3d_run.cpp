// nuc3d_run: the reference's single-box driver on the B200 path.
//
// Reads a case directory the way NUC3d does (inp/block.in, inp/Method.in,
// inp/PhysModel.in, inp/IOController.in; block.cpp:36-100,
// fieldOperator.cpp:21-125, physicsModel.cpp:66-156, IOcontroller.cpp:10-60),
// builds the initial state (Benchmark 2: Taylor-Green, 3: decaying isotropic
// turbulence, both generated on the device; startStep > 0: the restart file
// flowData/NUC3d_step_<startStep>_ID_0.bin, block.cpp:640-671), then runs
// singleBlock::solvePDE's loop (singleBlock.cpp:50-68): one TVD-RK3 step per
// iteration while time <= tl and step < endStep, the status line of
// block::printStatus (block.cpp:217-220), restart files every saveStep
// (block.cpp:609-638; with IOController "Tecplot yes" also the Tecplot file
// flowData/NUC3d_step_<step>_id_0.dat, block.cpp:553-607) and, every
// postStep, the solveQ statistics appended to
// enstrophy.dat and turb_para.dat (postproc.cpp:888-927) and the solveFFT
// shell spectra in flowDataTemp/power_shell_<step>_<name>.dat.
//
// Only the C ABI in include/nuc3d_b200.h is used.  One process, one box,
// periodic, process topology 1 1 1 (there is no MPI on this path).
// PhysModel.in Forcing None, Const (the spectral shell forcing) or Band (the
// band forcing at a fixed injection rate, this library's own keyword).
//
//   nuc3d_run [case_dir] [--precision fp64|mixed] [--seed S] [--check-decks]
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "nuc3d_b200.h"

namespace {

struct Case {
    nuc3d_box_desc desc{};
    std::map<std::string, double> io;    // IOController.in
    std::map<std::string, std::string> out;  // IOController.in output switches (yes/no)
    std::map<std::string, double> phys;  // PhysModel.in key/value part
    double x0 = 0, y0 = 0, z0 = 0;
};

[[noreturn]] void die(const std::string &msg) {
    std::cerr << "nuc3d_run: " << msg << std::endl;
    std::exit(1);
}

std::vector<std::string> words(const std::string &path, bool required) {
    std::ifstream f(path);
    if (!f) {
        if (required) die("File '" + path + "' does not exist!");
        return {};
    }
    std::vector<std::string> w;
    std::string s;
    while (f >> s) w.push_back(s);
    return w;
}

// fieldOperator3d::setMethodIvs* (fieldOperator.cpp:128-189): every scheme
// string the reference registers is on this path; a string it does not know
// falls back to weno5js, as the reference's does.
int scheme_id(const std::string &s) {
    if (s == "weno5js") return NUC3D_WENO5JS;
    if (s == "weno5z") return NUC3D_WENO5Z;
    if (s == "crweno5") return NUC3D_CRWENO5;
    if (s == "weno7js") return NUC3D_WENO7JS;
    if (s == "hccs") return NUC3D_HCCS;
    if (s == "hccs77") return NUC3D_HCCS77;
    if (s == "hccs78") return NUC3D_HCCS78;
    if (s == "weno3js") return NUC3D_WENO3JS;
    if (s == "upwind1st") return NUC3D_UPWIND1ST;
    return NUC3D_WENO5JS;
}

Case read_case(const std::string &dir) {
    Case c;
    nuc3d_box_desc_default(&c.desc);
    const std::string inp = dir + "/inp/";
    // block.in: npx npy npz / nx ny nz (global) / lx ly lz / x0 y0 z0 (block.cpp:49-70)
    auto b = words(inp + "block.in", true);
    if (b.size() < 9) die("block.in needs the topology, the mesh size and the box lengths");
    if (b[0] != "1" || b[1] != "1" || b[2] != "1")
        die("the B200 path runs one box per process (topology 1 1 1)");
    c.desc.nx = std::atoi(b[3].c_str());
    c.desc.ny = std::atoi(b[4].c_str());
    c.desc.nz = std::atoi(b[5].c_str());
    c.desc.lx = std::atof(b[6].c_str());
    c.desc.ly = std::atof(b[7].c_str());
    c.desc.lz = std::atof(b[8].c_str());
    if (b.size() >= 12) {
        c.x0 = std::atof(b[9].c_str());
        c.y0 = std::atof(b[10].c_str());
        c.z0 = std::atof(b[11].c_str());
    }
    // Method.in key/value (fieldOperator.cpp:21-125)
    std::map<std::string, std::string> method = {{"scheme_x_ivs", "weno5js"},
                                                 {"scheme_y_ivs", "weno5js"},
                                                 {"scheme_z_ivs", "weno5js"},
                                                 {"scheme_x_vis", "cd6"},
                                                 {"scheme_y_vis", "cd6"},
                                                 {"scheme_z_vis", "cd6"},
                                                 {"scheme_time", "RK3"}};
    auto m = words(inp + "Method.in", true);
    for (size_t i = 0; i + 1 < m.size(); i += 2)
        if (method.count(m[i])) method[m[i]] = m[i + 1];
    c.desc.scheme[0] = scheme_id(method["scheme_x_ivs"]);
    c.desc.scheme[1] = scheme_id(method["scheme_y_ivs"]);
    c.desc.scheme[2] = scheme_id(method["scheme_z_ivs"]);
    // fieldOperator3d::setDiffMethod* (fieldOperator.cpp:301-375): cd8, cd6
    // or cd2; any other string is cd6
    const char *vis_keys[3] = {"scheme_x_vis", "scheme_y_vis", "scheme_z_vis"};
    for (int d = 0; d < 3; ++d) {
        const std::string &v = method[vis_keys[d]];
        c.desc.vis_scheme[d] = v == "cd8" ? NUC3D_CD8 : (v == "cd2" ? NUC3D_CD2 : NUC3D_CD6);
    }
    if (method["scheme_time"] != "RK3") die("scheme_time " + method["scheme_time"] + ": only RK3");
    // PhysModel.in: six positional "key value" lines, then key/value pairs
    // (physicsModel.cpp:66-156); unknown keys stop the reference
    auto p = words(inp + "PhysModel.in", true);
    if (p.size() < 12) die("PhysModel.in needs its six positional lines");
    const std::string riemann = p[5], model = p[7], visc = p[9], forcing = p[11];
    // physicsModel.cpp:16-20 names; an unknown name makes the reference warn
    // and then compute no split at all (:88-93, :425-433), so it stops here
    if (riemann == "LF")
        c.desc.riemann = NUC3D_RIEMANN_LF;
    else if (riemann == "AUSM")
        c.desc.riemann = NUC3D_RIEMANN_AUSM;
    else if (riemann == "AUSMp")
        c.desc.riemann = NUC3D_RIEMANN_AUSMP;
    else
        die("Riemann Solver name " + riemann + " does not exist (LF, AUSM, AUSMp)");
    // "Band" is this library's band forcing at a fixed injection rate (not a
    // reference keyword)
    if (forcing != "None" && forcing != "Const" && forcing != "Band")
        die("Forcing " + forcing + ": only None, Const and Band are on the B200 path");
    c.desc.forcing = forcing == "Const"  ? NUC3D_FORCING_CONST
                     : forcing == "Band" ? NUC3D_FORCING_BAND
                                         : NUC3D_FORCING_NONE;
    if (model == "NavierStokes3d")
        c.desc.pde_model = NUC3D_NAVIERSTOKES3D;
    else if (model == "Euler3d")
        c.desc.pde_model = NUC3D_EULER3D;
    else
        die("Model Name:" + model + " does not exist!");
    c.desc.visc_model = visc == "Constant" ? NUC3D_VISC_CONSTANT : NUC3D_VISC_SUTHERLAND;
    c.phys = {{"Reynolds", 1000.0}, {"Mach", 0.5}, {"Pt", 0.72}, {"Gamma", 1.4},
              {"T_ref", 110.4}, {"T_inf", 288.0}, {"T_wall", 1.0}, {"Mach_t", 0.3},
              {"k_peak", 8.0}, {"Rossby", 0.0}, {"x_center", 3.1415926}, {"y_center", 3.1415926},
              {"z_center", 0.0}, {"well_rad", 1.0}, {"Forcing_amplitude", 0.01},
              {"Forcing_amplitude_hel", 0.01}, {"Forcing_wave_k", 1.0}};
    for (size_t i = 12; i + 1 < p.size(); i += 2) {
        if (p[i] == "Coriolis" || p[i] == "Centrifugal") {
            if (p[i + 1] != "no") die(p[i] + " source is not on the B200 path");
            continue;
        }
        if (!c.phys.count(p[i])) die("word " + p[i] + " does not exist");
        c.phys[p[i]] = std::atof(p[i + 1].c_str());
    }
    c.desc.reynolds = c.phys["Reynolds"];
    c.desc.mach = c.phys["Mach"];
    c.desc.prandtl = c.phys["Pt"];
    c.desc.gamma = c.phys["Gamma"];
    c.desc.t_ref = c.phys["T_ref"];
    c.desc.t_inf = c.phys["T_inf"];
    c.desc.forcing_amp = c.phys["Forcing_amplitude"];
    c.desc.forcing_hel = c.phys["Forcing_amplitude_hel"];
    c.desc.forcing_k = c.phys["Forcing_wave_k"];
    // IOController.in key/value (IOcontroller.cpp:10-60)
    c.io = {{"startStep", 0}, {"endStep", 100000}, {"postStep", 1}, {"saveStep", 1000},
            {"postSaveStep", 100}, {"Benchmark", 0}, {"cfl", 0.5}, {"tl", 0.0}, {"dt", 0.01}};
    // block::Output's switches (block.cpp:241-262); the restart file is
    // written at every save whatever "Binary" says (this driver restarts
    // from it), the Tecplot file only when "Tecplot" is "yes"
    c.out = {{"Binary", "no"}, {"Tecplot", "yes"}, {"PostProc", "no"}};
    auto io = words(inp + "IOController.in", false);
    for (size_t i = 0; i + 1 < io.size(); i += 2) {
        if (c.io.count(io[i])) c.io[io[i]] = std::atof(io[i + 1].c_str());
        if (c.out.count(io[i])) c.out[io[i]] = io[i + 1];
    }
    return c;
}

std::string restart_name(const std::string &dir, long long step) {
    return dir + "/flowData/NUC3d_step_" + std::to_string(step) + "_ID_0.bin";
}

// block.cpp:609-638: the time, then the five conserved fields, x-fastest
void write_restart(const std::string &path, double time, const std::vector<double> &q, long long n) {
    std::ofstream f(path, std::ios::binary);
    if (!f) die("cannot write " + path);
    f.write(reinterpret_cast<const char *>(&time), sizeof time);
    f.write(reinterpret_cast<const char *>(q.data()), (std::streamsize)(sizeof(double) * 5 * n));
}

double read_restart(const std::string &path, std::vector<double> &q, long long n) {
    std::ifstream f(path, std::ios::binary);
    if (!f) die("restart file '" + path + "' does not exist");
    double time = 0;
    f.read(reinterpret_cast<char *>(&time), sizeof time);
    f.read(reinterpret_cast<char *>(q.data()), (std::streamsize)(sizeof(double) * 5 * n));
    if (!f) die("restart file '" + path + "' is shorter than the mesh");
    return time;
}

// block::outputQ_tecplot (block.cpp:553-607): Tecplot ASCII, BLOCK packing;
// the mesh vertices x, y, z ((nx+1)(ny+1)(nz+1) each, block::getXYZ,
// block.cpp:103-140) then the cell-centred rho, u, v, w, pressure,
// temperature, e, sound_speed of physicsModel::con2prim
// (physicsModel.cpp:324-356), x fastest, one value per line with 12
// significant digits (utilities.cpp:47-61).
void write_tecplot(const std::string &path, const Case &c, const std::vector<double> &q,
                   long long n) {
    std::ofstream f(path);
    if (!f) die("cannot write " + path);
    const int nx = c.desc.nx, ny = c.desc.ny, nz = c.desc.nz;
    const char *names[8] = {"rho", "u", "v", "w", "pressure", "temperature", "e", "sound_speed"};
    f << "title=NUC3d\n"
      << "variables=x,y,z";
    for (const char *v : names) f << "," << v;
    f << "\n Zone I = " << nx + 1 << ", J= " << ny + 1 << ", K=" << nz + 1
      << "\n DATAPACKING=BLOCK, VARLOCATION=([4-11]=CELLCENTERED)\n";
    f << std::setprecision(12);
    const double d[3] = {c.desc.lx / nx, c.desc.ly / ny, c.desc.lz / nz};
    const double o[3] = {c.x0, c.y0, c.z0};
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k <= nz; ++k)
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i <= nx; ++i) {
                    const int ijk[3] = {i, j, k};
                    f << d[a] * ijk[a] - o[a] << "\n";
                }
    const double gamma = c.desc.gamma, mach = c.desc.mach;
    for (int v = 0; v < 8; ++v)
        for (long long m = 0; m < n; ++m) {
            const double rho = q[m], u = q[n + m] / rho, vv = q[2 * n + m] / rho,
                         w = q[3 * n + m] / rho, E = q[4 * n + m];
            const double p = std::fabs((E - 0.5 * rho * (u * u + vv * vv + w * w)) * (gamma - 1.0));
            double val;
            switch (v) {
                case 0: val = rho; break;
                case 1: val = u; break;
                case 2: val = vv; break;
                case 3: val = w; break;
                case 4: val = p; break;
                case 5: val = gamma * mach * mach * p / rho; break;
                case 6: val = p / rho / (gamma - 1.0); break;
                default: val = std::sqrt(gamma * p / rho); break;
            }
            f << val << "\n";
        }
    if (!f) die("write failed: " + path);
}

void check(int rc, const char *what) {
    if (rc != NUC3D_OK) die(std::string(what) + ": " + nuc3d_last_error());
}

}  // namespace

// postproc::solveFFT's shell spectra (postproc.cpp:931-1184) written as
// fft::solveShell writes them (fft.cpp:449-472): one file per spectrum,
// flowDataTemp/power_shell_<step>_<name>.dat, lines "i E_i E_i/sum(E)".
void write_spectra(nuc3d_ctx *ctx, const std::string &dir, long long step) {
    static const char *names[NUC3D_SPECTRA] = {"kin", "kinc", "kins", "kinl", "kinr",
                                               "hel", "ens", "den", "pre"};
    int kmax = 0;
    check(nuc3d_spectra(ctx, nullptr, &kmax), "nuc3d_spectra");
    std::vector<double> sp((size_t)NUC3D_SPECTRA * kmax);
    check(nuc3d_spectra(ctx, sp.data(), &kmax), "nuc3d_spectra");
    mkdir((dir + "/flowDataTemp").c_str(), 0755);
    for (int s = 0; s < NUC3D_SPECTRA; ++s) {
        const double *e = sp.data() + (size_t)s * kmax;
        double total = 0.0;
        for (int i = 0; i < kmax; ++i) total += e[i];
        std::ofstream f(dir + "/flowDataTemp/power_shell_" + std::to_string(step) + "_" +
                        names[s] + ".dat");
        for (int i = 0; i < kmax; ++i)
            f << std::setprecision(12) << i << " " << e[i] << " " << e[i] / total << "\n";
        f << std::endl;
    }
}

int main(int argc, char **argv) {
    std::string dir = ".";
    int precision = NUC3D_FP64;
    unsigned long long seed = 0;
    bool check_only = false;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--precision" && i + 1 < argc) {
            std::string v = argv[++i];
            precision = v == "mixed" ? NUC3D_MIXED : NUC3D_FP64;
        } else if (a == "--seed" && i + 1 < argc) {
            seed = std::strtoull(argv[++i], nullptr, 10);
        } else if (a == "--check-decks") {
            check_only = true;
        } else if (a == "-h" || a == "--help") {
            std::cout << "usage: nuc3d_run [case_dir] [--precision fp64|mixed] [--seed S] "
                         "[--check-decks]\n";
            return 0;
        } else {
            dir = a;
        }
    }
    Case c = read_case(dir);
    c.desc.precision = precision;
    const long long n = (long long)c.desc.nx * c.desc.ny * c.desc.nz;
    if (check_only) {
        std::cout << std::setprecision(17) << "nx " << c.desc.nx << " ny " << c.desc.ny << " nz "
                  << c.desc.nz << " lx " << c.desc.lx << " ly " << c.desc.ly << " lz " << c.desc.lz
                  << " scheme " << c.desc.scheme[0] << " " << c.desc.scheme[1] << " "
                  << c.desc.scheme[2] << " pde " << c.desc.pde_model << " visc "
                  << c.desc.visc_model << " gamma " << c.desc.gamma << " mach " << c.desc.mach
                  << " reynolds " << c.desc.reynolds << " prandtl " << c.desc.prandtl
                  << " t_ref " << c.desc.t_ref << " t_inf " << c.desc.t_inf << " forcing "
                  << c.desc.forcing << " forcing_amp " << c.desc.forcing_amp << " forcing_hel "
                  << c.desc.forcing_hel << " forcing_k " << c.desc.forcing_k << " riemann "
                  << c.desc.riemann << " vis " << c.desc.vis_scheme[0] << " "
                  << c.desc.vis_scheme[1] << " " << c.desc.vis_scheme[2] << " cfl "
                  << c.io["cfl"] << " endStep " << c.io["endStep"] << " tl " << c.io["tl"]
                  << std::endl;
        return 0;
    }
    if (c.x0 != 0.0 || c.y0 != 0.0 || c.z0 != 0.0)
        die("the device initial states use origin 0 0 0");
    nuc3d_ctx *ctx = nullptr;
    check(nuc3d_ctx_create(&c.desc, nullptr, &ctx), "nuc3d_ctx_create");
    std::vector<double> q((size_t)(5 * n));
    double *qp[5];
    for (int e = 0; e < 5; ++e) qp[e] = q.data() + e * n;
    const long long start = (long long)c.io["startStep"];
    double time = 0.0;
    long long step = start;
    if (start == 0) {
        nuc3d_init_desc init{};
        const int bench = (int)c.io["Benchmark"];
        if (bench == 2) {
            init.kind = NUC3D_INIT_TGV;
        } else if (bench == 3) {
            init.kind = NUC3D_INIT_HIT;
            init.seed = seed;
            init.k_peak = c.phys["k_peak"];
            init.mach_t = c.phys["Mach_t"];
        } else {
            die("Benchmark " + std::to_string(bench) + ": the B200 driver starts from 2 (Taylor-Green) "
                "or 3 (isotropic turbulence), or from a restart (startStep > 0)");
        }
        check(nuc3d_init_state(ctx, &init, nullptr), "nuc3d_init_state");
    } else {
        time = read_restart(restart_name(dir, start), q, n);
        const double *cq[5] = {qp[0], qp[1], qp[2], qp[3], qp[4]};
        check(nuc3d_set_state_host(ctx, cq), "nuc3d_set_state_host");
    }
    mkdir((dir + "/flowData").c_str(), 0755);
    const double cfl = c.io["cfl"], tl = c.io["tl"];
    const long long end = (long long)c.io["endStep"];
    const long long save = std::max(1LL, (long long)c.io["saveStep"]);
    const long long post = (long long)c.io["postStep"];
    auto output = [&]() {
        check(nuc3d_get_state_host(ctx, qp), "nuc3d_get_state_host");
        write_restart(restart_name(dir, step), time, q, n);
        if (c.out["Tecplot"] == "yes")
            write_tecplot(dir + "/flowData/NUC3d_step_" + std::to_string(step) + "_id_0.dat", c,
                          q, n);
    };
    std::cout << "Start solving......\n";
    while (time <= tl && step < end) {
        double dt = 0, res = 0;
        auto t0 = std::chrono::steady_clock::now();
        check(nuc3d_step(ctx, 1, cfl, &dt, &res), "nuc3d_step");
        double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        ++step;
        time += dt;
        std::cout << std::setprecision(6) << "========step = " << step << "\n time = " << time
                  << ", dt = " << dt << ", residual = " << res << ", CPU time = " << wall
                  << "(s) " << std::endl;
        if (post > 0 && step % post == 0) {
            double st[NUC3D_STATS];
            check(nuc3d_stats(ctx, st), "nuc3d_stats");
            std::ofstream fq(dir + "/enstrophy.dat", std::ios::app), ft(dir + "/turb_para.dat", std::ios::app);
            fq << std::setprecision(12) << step << " " << time;
            for (int i = 0; i < 16; ++i) fq << " " << st[i];
            fq << "\n";
            ft << std::setprecision(12) << step << " " << time;
            for (int i = 16; i < 25; ++i) ft << " " << st[i];
            ft << "\n";
            write_spectra(ctx, dir, step);
        }
        if (step % save == 0) output();
    }
    output();
    std::cout << "Calculation finished!!" << std::endl;
    check(nuc3d_ctx_destroy(ctx), "nuc3d_ctx_destroy");
    return 0;
}
