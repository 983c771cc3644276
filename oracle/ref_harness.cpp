// Driver around the reference's own serial C++ hot path -- TEST INFRASTRUCTURE.
//
// Built by oracle/Makefile from the reference sources where they lie (this
// file is compiled with the reference tree on the include path; no reference
// source is copied).  It reads the reference's binary inputs, runs the
// reference's routines and dumps their outputs as raw float64 files:
//
//   hfem_ref assemble <in> <out> [nelem_dump]
//       getQ on every element (dgsolvers.cpp:464-474), assembleLinearSystem
//       (globalassembly.cpp:423-556); writes udg, Hg, Rg, Rr, DinvRu, DinvF,
//       rnorm, and the pre-condensation blocks of the first nelem_dump elements
//       (assembleElementMatrixVector, elementassembly.cpp:1481-1499).
//   hfem_ref newton <in> <out> <maxiter> <precond> <restart> <gmres_tol>
//       the reference Newton driver solveNonlinearProblem (dgsolvers.cpp:106-205)
//       after getQ; writes the final udg, uh and the residual / GMRES histories.
//   hfem_ref dirk <in> <out> <nsteps> <precond> <restart> <gmres_tol>
//       nsteps time steps of the reference's own DIRK driver solveUnsteadyProblem
//       (dgsolvers.cpp:221-444; tableau, dt and Newton limits from the app file),
//       one step per call (app.dt holds one step); writes UDG after getQ and after
//       every step, nsteps + 1 states back to back.
//   hfem_ref timing <in> <nelem> <reps>
//       times assembleLinearSystem over the first nelem elements; prints JSON.
//
// For time-dependent inputs (app.flag[0] = 1) the source SH = fc_u * UDG (u part)
// is set as the first DIRK stage does (dgsolvers.cpp:323-348).
#include <string>
#include <fstream>
#include <sstream>
#include <iostream>
#include <vector>
#include <algorithm>
#include <numeric>
#include <chrono>
#include <math.h>
#include <stdlib.h>

using namespace std;

#include "preprocessing/digasopre.h"
#include "preprocessing/preprocessing.cpp"
#include "assembly/assembly.cpp"
#include "solvers/dgsolvers.cpp"
#include "ref_closed.cpp"

static void dump(const string& path, const double* p, size_t n)
{
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
    fwrite(p, sizeof(double), n, f);
    fclose(f);
}

static vector<Int> ndims_of(meshstruct& mesh, masterstruct& m, appstruct& app, sysstruct& sys)
{
    vector<Int> nd(100, 0);
    nd[0] = app.nd; nd[1] = app.ncd; nd[2] = mesh.nfemax; nd[3] = mesh.nvemax; nd[4] = mesh.nvfmax;
    nd[5] = mesh.ne; nd[6] = mesh.nf; nd[7] = mesh.nv; nd[8] = mesh.ndofuh; nd[9] = mesh.npemax;
    nd[10] = mesh.npfmax; nd[11] = mesh.nmemax; nd[12] = mesh.nmfmax; nd[13] = mesh.ngemax;
    nd[14] = mesh.ngfmax; nd[15] = app.porder[0]; nd[16] = app.porder[0]; nd[17] = app.dirkOrder;
    nd[18] = app.dirkStage; nd[19] = app.nc; nd[20] = app.ncu; nd[21] = app.ncq; nd[22] = app.ncp;
    nd[23] = app.nch; nd[31] = sys.numEntities; nd[32] = sys.numBlocks; nd[33] = sys.maxBlocksPerRow;
    nd[34] = sys.blkSize; nd[35] = sys.BJ_nrows; nd[39] = sys.nproc; nd[75] = mesh.ncfmax;
    return nd;
}

struct Ctx {
    appstruct app;
    vector<masterstruct> master;
    meshstruct mesh;
    solstruct sol;
    sysstruct sys;
    elemstruct elem;
    tempstruct temp;
    vector<Int> ndims;
};

static void setup(Ctx& c, const string& in)
{
    c.app.filein = in;
    c.app.fileout = in + "out";
    c.app.my_rank = 0; c.app.nproc = 1; c.app.debugmode = 0;
    c.sys.my_rank = 0; c.sys.noThreads = 1;
    c.mesh.my_rank = 0;
    preprocessing(c.mesh, c.master, c.app, c.sol, c.elem, c.sys, c.temp, in, c.app.fileout);
    c.elem.my_rank = 0;
    masterstruct& m = c.master[c.mesh.elementtype[0]];
    c.ndims = ndims_of(c.mesh, m, c.app, c.sys);
    const Int npv = m.npv, nc = c.app.nc, ncu = c.app.ncu, ne = c.mesh.ne;
    if (c.app.tdep == 1) {
        for (Int e = 0; e < ne; e++)
            for (Int j = 0; j < nc; j++)
                for (Int k = 0; k < npv; k++) {
                    const size_t idx = k + j * npv + (size_t)e * npv * nc;
                    c.sol.SH[idx] = (j < ncu) ? c.app.fc_u * c.sol.UDG[idx] : 0.0;
                }
    }
    if (c.app.flag_q == 1)
      for (Int ie = 0; ie < ne; ie++)
        getQ(c.elem, c.mesh, m, c.app, c.sol, c.temp, &c.sol.UDG[ie * npv * nc],
             &c.sol.UDG[ie * npv * nc + npv * ncu], &c.sol.UH[0], &c.sol.SH[ie * npv * nc + npv * ncu], ie);
}

int main(int argc, char** argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: hfem_ref assemble|newton|timing <inprefix> ...\n");
        return 1;
    }
    string mode = argv[1], in = argv[2];
    Ctx c;
    setup(c, in);
    masterstruct& m = c.master[c.mesh.elementtype[0]];
    const Int npv = m.npv, ncu = c.app.ncu, nch = c.app.nch, ne = c.mesh.ne;
    const Int ndf = m.ndf, n = npv * ncu, nb = nch * ndf;

    if (mode == "assemble") {
        string out = argv[3];
        Int ndump = (argc > 4) ? atoi(argv[4]) : 0;
        dump(out + "udg.bin", &c.sol.UDG[0], c.sol.UDG.size());
        assembleLinearSystem(c.sys, &c.elem, c.mesh, m, c.sol, c.app, &c.temp);
        dump(out + "Hg.bin", &c.sys.Hg[0], c.sys.Hg.size());
        dump(out + "Rg.bin", &c.sys.Rg[0], c.sys.Rg.size());
        dump(out + "Rr.bin", &c.sys.r[0], c.sys.r.size());
        dump(out + "DinvRu.bin", &c.sol.DinvRu[0], (size_t)n * ne);
        dump(out + "DinvF.bin", &c.sol.DinvF[0], (size_t)n * nb * ne);
        dump(out + "rnorm.bin", &c.sol.rNorm, 1);
        vector<double> D, F, K, H, Ru, Rh;
        double et[32] = {0};
        for (Int ie = 0; ie < min(ndump, ne); ie++) {
            assembleElementMatrixVector(c.elem, c.mesh, m, c.app, c.sol, c.temp, ie, et);
            D.insert(D.end(), &c.elem.BD[0], &c.elem.BD[0] + n * n);
            F.insert(F.end(), &c.elem.F[0], &c.elem.F[0] + n * nb);
            K.insert(K.end(), &c.elem.GK[0], &c.elem.GK[0] + nb * n);
            H.insert(H.end(), &c.elem.H[0], &c.elem.H[0] + nb * nb);
            Ru.insert(Ru.end(), &c.elem.Ru[0], &c.elem.Ru[0] + n);
            Rh.insert(Rh.end(), &c.elem.Rh[0], &c.elem.Rh[0] + nb);
        }
        if (ndump > 0) {
            dump(out + "eD.bin", D.data(), D.size());
            dump(out + "eF.bin", F.data(), F.size());
            dump(out + "eK.bin", K.data(), K.size());
            dump(out + "eH.bin", H.data(), H.size());
            dump(out + "eRu.bin", Ru.data(), Ru.size());
            dump(out + "eRh.bin", Rh.data(), Rh.size());
        }
        return 0;
    }
    if (mode == "newton") {
        string out = argv[3];
        c.sys.NewtonMaxiter = c.sys.trueNewtonMaxiter = atoi(argv[4]);
        c.sys.preconditioner = atoi(argv[5]);
        c.sys.restart = atoi(argv[6]);
        c.sys.tol = atof(argv[7]);
        if (argc > 8) c.sys.reorderMethod = atoi(argv[8]);
        g_sol = &c.sol;
        Int conv[1] = {0};
        solveNonlinearProblem(c.sys, &c.elem, c.mesh, m, c.sol, c.app, &c.temp, &c.ndims[0], conv);
        g_newton_rnorm.push_back(c.sol.rNorm);
        dump(out + "udg.bin", &c.sol.UDG[0], c.sol.UDG.size());
        dump(out + "uh.bin", &c.sol.UH[0], c.sol.UH.size());
        dump(out + "rnorm_hist.bin", g_newton_rnorm.data(), g_newton_rnorm.size());
        vector<double> its(g_gmres_iters.begin(), g_gmres_iters.end());
        dump(out + "gmres_iters.bin", its.data(), its.size());
        dump(out + "gmres_hist.bin", g_gmres_hist.data(), g_gmres_hist.size());
        return 0;
    }
    if (mode == "dirk") {
        string out = argv[3];
        const Int nsteps = atoi(argv[4]);
        c.sys.preconditioner = atoi(argv[5]);
        c.sys.restart = atoi(argv[6]);
        c.sys.tol = atof(argv[7]);
        g_sol = &c.sol;
        vector<double> states(c.sol.UDG.begin(), c.sol.UDG.end());
        for (Int s = 0; s < nsteps; s++) {
            solveUnsteadyProblem(c.sys, &c.elem, c.mesh, m, c.sol, c.app, &c.temp, &c.ndims[0]);
            states.insert(states.end(), c.sol.UDG.begin(), c.sol.UDG.end());
        }
        dump(out + "udg_steps.bin", states.data(), states.size());
        return 0;
    }
    if (mode == "timing") {
        Int nel = atoi(argv[3]), reps = atoi(argv[4]);
        if (nel > 0 && nel < ne) c.mesh.ne = nel;
        assembleLinearSystem(c.sys, &c.elem, c.mesh, m, c.sol, c.app, &c.temp);   // warm-up
        auto t0 = chrono::steady_clock::now();
        for (Int r = 0; r < reps; r++)
            assembleLinearSystem(c.sys, &c.elem, c.mesh, m, c.sol, c.app, &c.temp);
        double s = chrono::duration<double>(chrono::steady_clock::now() - t0).count();
        printf("{\"elements\": %d, \"reps\": %d, \"seconds\": %.6f, \"elems_per_s\": %.3f}\n",
               (int)c.mesh.ne, (int)reps, s, (double)c.mesh.ne * reps / s);
        return 0;
    }
    fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 1;
}
