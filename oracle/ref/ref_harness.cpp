// C entry surface over the reference's OWN classes, compiled from the
// reference's sources where they lie.  TEST INFRASTRUCTURE ONLY: this is the
// checker that pins the C restatement in oracle/nuc3d_oracle.c and generates
// the golden fixtures under tests/golden/.  It is never linked into the
// product and never shipped.
//
// What each entry point drives (reference file:line):
//   ref_reconstruct   weno5js / weno5z / crweno5 / weno7js / hccs ::interpolationInner +
//                     interpolationBoundaryL/R          (weno5js.cpp:19-628,
//                     weno5z.cpp:18-637, crweno5.cpp:25-837); output = n+1 faces
//   ref_cd6           centraldifference6th::differentialInner/BoundaryL/R
//                     (centraldifference6th.cpp:16-186)
//   ref_cd            centraldifference6th / 2nd / 8th (scheme 0 / 1 / 2) with a
//                     given tilesize (centraldifference2nd.cpp:16-146,
//                     centraldifference8th.cpp:22-205)
//   ref_rk3_stage     tvdrk3rd::integrationAll (TVD-RK3.cpp:16-157)
//   ref_split         physicsModel::solve (con2prim) + solveRiemann (RiemannLF)
//                     (physicsModel.cpp:158-165, 276-357, 436-680)
//   ref_rhs           one NaiverStokesData3d::solve / EulerData3D::solve
//                     (NaiverStokes3d.cpp:37-73, euler3d.cpp:260-277)
//   ref_run_steps     block::solve's stage loop (block.cpp:191-215) for
//                     nsteps steps, PDEData3d::solve (PDEData3d.cpp:155-213)
//   ref_stats         postproc::solveQ (postproc.cpp:736-930): the averages it
//                     keeps and the turb_para.dat line it writes
//   ref_spectra       postproc::solveFFT (postproc.cpp:931-1184): the nine
//                     shell spectra it writes (FFTs through the DFT stand-in)
//
// The solver classes read their decks from ./inp relative to the working
// directory (fieldOperator.cpp:34, physicsModel.cpp:67), so the whole-step
// entry points chdir into a caller-prepared directory first.

#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "NaiverStokes3d.h"
#include "PDEData3d.hpp"
#include "TVD-RK3.h"
#include "bufferData.hpp"
#include "centraldifference2nd.hpp"
#include "centraldifference6th.h"
#include "centraldifference8th.hpp"
#include "crweno5.hpp"
#include "euler3d.h"
#include "fft.h"
#include "fieldOperator.h"
#include "hccs.hpp"
#include "hccs77.hpp"
#include "hccs78.hpp"
#include "upwind1st.hpp"
#include "weno3js.hpp"
#include "physicsModel.h"
#include "weno5js.h"
#include "weno5z.hpp"
#include "weno7js.hpp"
// solveQ is declared under `private:`; the harness calls it directly
// (access only, the class layout is unchanged).
#define private public
#include "postproc.hpp"
#undef private

#include <cstdio>
#include <fstream>

using nuc3d::Field;
using nuc3d::VectorField;

namespace {

void to_field(const double *src, Field &f) {
    std::memcpy(f.getDataPtr(), src, sizeof(double) * static_cast<size_t>(f.getSize()));
}
void from_field(const Field &f, double *dst) {
    std::memcpy(dst, f.getDataPtr(), sizeof(double) * static_cast<size_t>(f.getSize()));
}

struct Cwd {
    std::string old;
    explicit Cwd(const char *dir) {
        char buf[4096];
        if (getcwd(buf, sizeof buf)) old = buf;
        if (chdir(dir) != 0) old.clear();
    }
    ~Cwd() {
        if (!old.empty()) (void)chdir(old.c_str());
    }
};

// One reference solver instance built the way block::initial builds it
// (block.cpp:36-100, 143-187), with the periodic single-rank topology.
struct RefSolver {
    nuc3d::MPIComunicator3d_nonblocking mpi;
    nuc3d::physicsModel phys;
    nuc3d::fieldOperator3d op;
    nuc3d::PDEData3d pde;
    std::shared_ptr<nuc3d::EulerData3D> flux;
    std::vector<nuc3d::bufferData> buffers;
    nuc3d::fft fft;
    VectorField xyz_center;

    RefSolver(int nx, int ny, int nz, double dx, double dy, double dz)
        : pde(nx, ny, nz, 5) {
        mpi.setTopo(1, 1, 1);
        fft.initFFT(mpi, nx, ny, nz);  // block.cpp initialises it for every run
        if (phys.getMyModelName() == "NavierStokes3d")
            flux = std::make_shared<nuc3d::NaiverStokesData3d>(nx, ny, nz, 5, dx, dy, dz);
        else
            flux = std::make_shared<nuc3d::EulerData3D>(nx, ny, nz, 5, dx, dy, dz);
        int bfsize = op.bufferSize_xi;
        if (op.bufferSize_eta > bfsize) bfsize = op.bufferSize_eta;
        if (op.bufferSize_zeta > bfsize) bfsize = op.bufferSize_zeta;
        for (int n = 0; n < 5; ++n) buffers.push_back(nuc3d::bufferData(nx, ny, nz, bfsize));
        for (int d = 0; d < 3; ++d) xyz_center.push_back(Field(nx, ny, nz));
    }
    void load(const double *const q[5]) {
        VectorField &Q = pde.getQ();
        for (int e = 0; e < 5; ++e) to_field(q[e], Q[e]);
    }
    void store(double *const q[5]) {
        VectorField &Q = pde.getQ();
        for (int e = 0; e < 5; ++e) from_field(Q[e], q[e]);
    }
    void rhs_eval() { flux->solve(pde, op, buffers, phys, mpi, fft, xyz_center); }
};

}  // namespace

// one differential scheme's inner and boundary passes over a field
template <typename S>
void run_differential(const Field &fin, double dx, const Field &fl, const Field &fr, Field &fout,
                      int tile) {
    S s;
    s.differentialInner(fin, dx, fout, tile);
    s.differentialBoundaryL(fin, dx, fl, fout, tile);
    s.differentialBoundaryR(fin, dx, fr, fout, tile);
}

extern "C" {

// scheme: 0 = weno5js, 1 = weno5z, 2 = crweno5, 3 = weno7js, 4 = hccs,
// 5 = hccs77, 6 = hccs78, 7 = weno3js, 8 = upwind1st.
// in: (nx,ny,nz); halos: (tile,ny,nz) with tile the scheme's bufferSize (3;
// 4 for weno7js and the hccs family, 2 for weno3js, 1 for upwind1st);
// out: (nx+1,ny,nz).  Reconstruction runs along the fastest axis.
int ref_reconstruct(int scheme, int upwind, int nx, int ny, int nz, const double *in,
                    const double *halo_l, const double *halo_r, double *out) {
    // bufferSize (fieldOperator.cpp:131-175)
    const int tile = scheme == 7 ? 2 : (scheme == 8 ? 1 : (scheme >= 3 ? 4 : 3));
    Field fin(nx, ny, nz), fl(tile, ny, nz), fr(tile, ny, nz), fout(nx + 1, ny, nz);
    to_field(in, fin);
    to_field(halo_l, fl);
    to_field(halo_r, fr);
    to_field(out, fout);
    if (scheme == 0) {
        nuc3d::weno5js s;
        s.interpolationInner(fin, upwind, fout, tile);
        s.interpolationBoundaryL(fin, fl, upwind, fout, tile);
        s.interpolationBoundaryR(fin, fr, upwind, fout, tile);
    } else if (scheme == 1) {
        nuc3d::weno5z s;
        s.interpolationInner(fin, upwind, fout, tile);
        s.interpolationBoundaryL(fin, fl, upwind, fout, tile);
        s.interpolationBoundaryR(fin, fr, upwind, fout, tile);
    } else if (scheme == 2) {
        nuc3d::crweno5 s;
        s.interpolationInner(fin, upwind, fout, tile);
        s.interpolationBoundaryL(fin, fl, upwind, fout, tile);
        s.interpolationBoundaryR(fin, fr, upwind, fout, tile);
    } else if (scheme == 3) {
        nuc3d::weno7js s;
        s.interpolationInner(fin, upwind, fout, tile);
        s.interpolationBoundaryL(fin, fl, upwind, fout, tile);
        s.interpolationBoundaryR(fin, fr, upwind, fout, tile);
    } else if (scheme == 4) {
        nuc3d::hccs s;
        s.interpolationInner(fin, upwind, fout, tile);
        s.interpolationBoundaryL(fin, fl, upwind, fout, tile);
        s.interpolationBoundaryR(fin, fr, upwind, fout, tile);
    } else if (scheme == 5) {
        nuc3d::hccs77 s;
        s.interpolationInner(fin, upwind, fout, tile);
        s.interpolationBoundaryL(fin, fl, upwind, fout, tile);
        s.interpolationBoundaryR(fin, fr, upwind, fout, tile);
    } else if (scheme == 6) {
        nuc3d::hccs78 s;
        s.interpolationInner(fin, upwind, fout, tile);
        s.interpolationBoundaryL(fin, fl, upwind, fout, tile);
        s.interpolationBoundaryR(fin, fr, upwind, fout, tile);
    } else if (scheme == 7) {
        nuc3d::weno3js s;
        s.interpolationInner(fin, upwind, fout, tile);
        s.interpolationBoundaryL(fin, fl, upwind, fout, tile);
        s.interpolationBoundaryR(fin, fr, upwind, fout, tile);
    } else if (scheme == 8) {
        nuc3d::upwind1st s;
        s.interpolationInner(fin, upwind, fout, tile);
        s.interpolationBoundaryL(fin, fl, upwind, fout, tile);
        s.interpolationBoundaryR(fin, fr, upwind, fout, tile);
    } else {
        return -1;
    }
    from_field(fout, out);
    return 0;
}

int ref_cd6(int nx, int ny, int nz, double dx, const double *in, const double *halo_l,
            const double *halo_r, double *out) {
    const int tile = 3;
    Field fin(nx, ny, nz), fl(tile, ny, nz), fr(tile, ny, nz), fout(nx, ny, nz);
    to_field(in, fin);
    to_field(halo_l, fl);
    to_field(halo_r, fr);
    nuc3d::centraldifference6th s;
    s.differentialInner(fin, dx, fout, tile);
    s.differentialBoundaryL(fin, dx, fl, fout, tile);
    s.differentialBoundaryR(fin, dx, fr, fout, tile);
    from_field(fout, out);
    return 0;
}

// halos are (tile, ny, nz); -1 where the scheme's stencil would read outside
// them (cd6 with tile < 3, cd8 with tile < 4)
int ref_cd(int scheme, int tile, int nx, int ny, int nz, double dx, const double *in,
           const double *halo_l, const double *halo_r, double *out) {
    const int reach = scheme == 1 ? 1 : (scheme == 2 ? 4 : 3);
    if (tile < reach || tile > 4 || nx < 2 * tile) return -1;
    Field fin(nx, ny, nz), fl(tile, ny, nz), fr(tile, ny, nz), fout(nx, ny, nz);
    to_field(in, fin);
    to_field(halo_l, fl);
    to_field(halo_r, fr);
    if (scheme == 0)
        run_differential<nuc3d::centraldifference6th>(fin, dx, fl, fr, fout, tile);
    else if (scheme == 1)
        run_differential<nuc3d::centraldifference2nd>(fin, dx, fl, fr, fout, tile);
    else if (scheme == 2)
        run_differential<nuc3d::centraldifference8th>(fin, dx, fl, fr, fout, tile);
    else
        return -1;
    from_field(fout, out);
    return 0;
}

// ui is updated in place, as in the reference.
int ref_rk3_stage(int stage, int n, double dt, const double *const rhs[5],
                  const double *const un[5], double *const ui[5]) {
    VectorField R(5, Field(n, 1, 1)), U(5, Field(n, 1, 1)), Ui(5, Field(n, 1, 1));
    for (int e = 0; e < 5; ++e) {
        to_field(rhs[e], R[e]);
        to_field(un[e], U[e]);
        to_field(ui[e], Ui[e]);
    }
    nuc3d::tvdrk3rd rk;
    rk.integrationAll(R, U, Ui, dt, stage);
    for (int e = 0; e < 5; ++e) from_field(Ui[e], ui[e]);
    return 0;
}

// con2prim + RiemannLF.  flux_l/flux_r: 15 arrays each, [dir*5+eq], in the
// reference's rotated layouts (xi: x-fastest; eta: (ny,nz,nx); zeta: (nz,nx,ny)).
// prim: 8 arrays (rho,u,v,w,p,T,e,c).  eig: 3 maxEigen values.
int ref_split(const char *workdir, int nx, int ny, int nz, const double *const q[5],
              double *const prim[8], double *const flux_l[15], double *const flux_r[15],
              double *eig) {
    Cwd cwd(workdir);
    RefSolver s(nx, ny, nz, 1.0, 1.0, 1.0);
    s.load(q);
    s.phys.solve(s.pde, s.flux.get());
    s.phys.solveRiemann(s.pde, s.flux.get());
    VectorField &W = s.flux->getPrimatives();
    VectorField &W0 = s.flux->getAcoustics();
    for (int e = 0; e < 5; ++e) from_field(W[e], prim[e]);
    for (int e = 0; e < 3; ++e) from_field(W0[e], prim[5 + e]);
    nuc3d::EulerFlux *fl[3] = {&s.flux->getFluxXi(), &s.flux->getFluxEta(),
                               &s.flux->getFluxZeta()};
    for (int d = 0; d < 3; ++d) {
        for (int e = 0; e < 5; ++e) {
            from_field(fl[d]->FluxL[e], flux_l[d * 5 + e]);
            from_field(fl[d]->FluxR[e], flux_r[d * 5 + e]);
        }
        eig[d] = fl[d]->maxEigen;
    }
    return 0;
}

// One RHS evaluation on q.  rhs: 5 arrays (x-fastest).  dt_local: the value
// the solver hands to PDEData3d::setDt.
int ref_rhs(const char *workdir, int nx, int ny, int nz, double dx, double dy, double dz,
            const double *const q[5], double *const rhs[5], double *dt_local) {
    Cwd cwd(workdir);
    RefSolver s(nx, ny, nz, dx, dy, dz);
    s.load(q);
    s.rhs_eval();
    VectorField &R = s.pde.getRHS();
    for (int e = 0; e < 5; ++e) from_field(R[e], rhs[e]);
    *dt_local = s.pde.dt_local;
    return 0;
}

// nsteps full TVD-RK3 steps; q is replaced by the final state.  dt[s] and
// res[s] receive the step's dt_global and residual (block.cpp:208-214).
int ref_run_steps(const char *workdir, int nx, int ny, int nz, double dx, double dy, double dz,
                  double cfl, int nsteps, double *const q[5], double *dt, double *res) {
    Cwd cwd(workdir);
    RefSolver s(nx, ny, nz, dx, dy, dz);
    s.load(q);
    for (int n = 0; n < nsteps; ++n) {
        int stage = 0;
        while (s.op.getSteps() != stage) {
            s.rhs_eval();
            s.pde.solve(s.op, s.mpi, cfl, stage++);
        }
        dt[n] = s.pde.getDt();
        res[n] = s.pde.getRes();
    }
    s.store(q);
    return 0;
}

// postproc::solveQ on q (istep 0, time 0).  out[0..15]: the 16 field
// averages of enstrophy.dat; out[16..24]: the turb_para.dat values; both read
// back from the files solveQ writes (12 significant digits).  The workdir
// needs inp/PostProc.in with SimutaneousData 1.
int ref_stats(const char *workdir, int nx, int ny, int nz, double dx, double dy, double dz,
              const double *const q[5], double *out) {
    Cwd cwd(workdir);
    RefSolver s(nx, ny, nz, dx, dy, dz);
    s.load(q);
    VectorField prim(5, Field(nx, ny, nz)), acou(3, Field(nx, ny, nz));
    s.phys.getPrim(s.pde.getQ(), prim, acou);
    nuc3d::postproc post(nx, ny, nz, dx, dy, dz);
    std::remove("enstrophy.dat");
    std::remove("turb_para.dat");
    post.solveQ(prim, acou, s.phys, s.op, s.buffers, s.mpi, 0, 0.0);
    double step, time;
    std::ifstream fq("enstrophy.dat");
    if (!(fq >> step >> time)) return -1;
    for (int i = 0; i < 16; ++i)
        if (!(fq >> out[i])) return -2;
    std::ifstream f("turb_para.dat");
    if (!(f >> step >> time)) return -3;
    for (int i = 0; i < 9; ++i)
        if (!(f >> out[16 + i])) return -4;
    return 0;
}

// postproc::solveTemporal's spectra (postproc.cpp:931-1184 with
// fft.cpp:182-572) on q: solveQ for the enstrophy and helicity fields, then
// solveFFT, which writes flowDataTemp/power_shell_0_<name>.dat per spectrum.
// out[s*kmax + i] = shell i of spectrum s in the order kin, kinc, kins, kinl,
// kinr, hel, ens, den, pre (12 significant digits, as written), kmax =
// min(nx, ny, nz)/2.  The FFTs run through the DFT stand-in for FFTW.
int ref_spectra(const char *workdir, int nx, int ny, int nz, double dx, double dy, double dz,
                const double *const q[5], double *out) {
    Cwd cwd(workdir);
    if (mkdir("flowDataTemp", 0755) != 0 && errno != EEXIST) return -1;
    RefSolver s(nx, ny, nz, dx, dy, dz);
    s.load(q);
    VectorField prim(5, Field(nx, ny, nz)), acou(3, Field(nx, ny, nz));
    s.phys.getPrim(s.pde.getQ(), prim, acou);
    nuc3d::postproc post(nx, ny, nz, dx, dy, dz);
    post.solveQ(prim, acou, s.phys, s.op, s.buffers, s.mpi, 0, 0.0);
    post.solveFFT(prim, acou, s.op, s.buffers, s.mpi, s.fft, 0, 0.0);
    const int kmax = std::min(std::min(nx, ny), nz) / 2;
    const char *names[9] = {"kin", "kinc", "kins", "kinl", "kinr", "hel", "ens", "den", "pre"};
    for (int sp = 0; sp < 9; ++sp) {
        std::ifstream f(std::string("flowDataTemp/power_shell_0_") + names[sp] + ".dat");
        for (int i = 0; i < kmax; ++i) {
            double idx, val, frac;
            if (!(f >> idx >> val >> frac) || (int)idx != i) return -2 - sp;
            out[sp * kmax + i] = val;
        }
    }
    return 0;
}

}  // extern "C"
