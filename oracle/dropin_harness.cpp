// The reference's own serial Newton driver running on the GPU through
// hfem_b200/shim/reference_shim.cpp -- TEST INFRASTRUCTURE (the drop-in check).
//
// Built by oracle/Makefile from the reference sources where they lie, like
// ref_harness.cpp, but with the reference's assembly, solution update and
// closed solver routines replaced by the shim and libhfem_b200.so:
// preprocessing/preprocessing.cpp and solvers/dgsolvers.cpp are compiled
// unchanged; assembly/assembly.cpp and solvers/solutionupdate.cpp are not
// compiled at all; dmdserial (closed) is the restatement in ref_dmdserial.cpp.
//
//   digasoser_b200 newton <in> <out> <maxiter> <precond> <restart> <gmres_tol>
//       getQ (through the shim) and solveNonlinearProblem (dgsolvers.cpp:106-205);
//       writes the final udg, uh and the residual history (the assembly residual
//       of every Newton iteration, then the final residual).
#include <string>
#include <fstream>
#include <sstream>
#include <iostream>
#include <vector>
#include <algorithm>
#include <numeric>
#include <math.h>
#include <stdlib.h>

using namespace std;

#include "preprocessing/digasopre.h"
#include "preprocessing/preprocessing.cpp"
#define __SOLUTIONUPDATE
#include "../hfem_b200/shim/reference_shim.cpp"
#include "solvers/dgsolvers.cpp"
#include "ref_dmdserial.cpp"

static void dump(const string& path, const double* p, size_t n)
{
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
    fwrite(p, sizeof(double), n, f);
    fclose(f);
}

int main(int argc, char** argv)
{
    if (argc < 8 || string(argv[1]) != "newton") {
        fprintf(stderr, "usage: digasoser_b200 newton <inprefix> <outprefix> <maxiter> <precond> <restart> <gmres_tol>\n");
        return 1;
    }
    const string in = argv[2], out = argv[3];
    appstruct app;
    vector<masterstruct> master;
    meshstruct mesh;
    solstruct sol;
    sysstruct sys;
    elemstruct elem;
    tempstruct temp;
    app.filein = in;
    app.fileout = in + "out";
    app.my_rank = 0; app.nproc = 1; app.debugmode = 0;
    sys.my_rank = 0; sys.noThreads = 1;
    mesh.my_rank = 0;
    preprocessing(mesh, master, app, sol, elem, sys, temp, in, app.fileout);
    elem.my_rank = 0;
    masterstruct& m = master[mesh.elementtype[0]];
    vector<Int> nd(100, 0);
    nd[2] = mesh.nfemax; nd[5] = mesh.ne; nd[6] = mesh.nf; nd[9] = mesh.npemax; nd[10] = mesh.npfmax;
    nd[19] = app.nc; nd[20] = app.ncu; nd[23] = app.nch; nd[75] = mesh.ncfmax;
    // time-dependent inputs: the first DIRK stage's source SH = fc_u UDG on u
    // (dgsolvers.cpp:323-348), as oracle/ref_harness.cpp sets it
    if (app.tdep == 1)
        for (Int e = 0; e < mesh.ne; e++)
            for (Int j = 0; j < app.nc; j++)
                for (Int k = 0; k < m.npv; k++) {
                    const size_t idx = k + j * m.npv + (size_t)e * m.npv * app.nc;
                    sol.SH[idx] = (j < app.ncu) ? app.fc_u * sol.UDG[idx] : 0.0;
                }
    sys.NewtonMaxiter = sys.trueNewtonMaxiter = atoi(argv[4]);
    sys.preconditioner = atoi(argv[5]);
    sys.restart = atoi(argv[6]);
    sys.tol = atof(argv[7]);
    // q from (u, uh), as solveProblem does before its solve (dgsolvers.cpp:464-474);
    // the residual call builds the GPU context from the structs
    computeResidualNorm(sys, &elem, mesh, m, sol, app, &temp);
    if (app.flag_q == 1)
        for (Int ie = 0; ie < mesh.ne; ie++)
            getQ(elem, mesh, m, app, sol, temp, &sol.UDG[ie * m.npv * app.nc],
                 &sol.UDG[ie * m.npv * app.nc + m.npv * app.ncu], &sol.UH[0],
                 &sol.SH[ie * m.npv * app.nc + m.npv * app.ncu], ie);
    Int conv[1] = {0};
    solveNonlinearProblem(sys, &elem, mesh, m, sol, app, &temp, &nd[0], conv);
    vector<double> hist = hfem_shim::g_rnorm_log;
    hist.push_back(sol.rNorm);
    dump(out + "udg.bin", &sol.UDG[0], sol.UDG.size());
    dump(out + "uh.bin", &sol.UH[0], sol.UH.size());
    dump(out + "rnorm_hist.bin", hist.data(), hist.size());
    return 0;
}
