// Reference-side binding of libhfem_b200: the routines of the reference's
// serial solver chain, with the reference's own signatures, implemented on the
// C ABI of include/hfem_b200.h.
//
// A host program built from the reference's sources (main/digasoser.cpp) uses
// this file in place of assembly/assembly.cpp, solvers/solutionupdate.cpp and
// the closed solver archives (gmres, computePreconditioner, computeOrdering);
// solvers/dgsolvers.cpp is compiled unchanged and its Newton and DIRK drivers
// run on the GPU through these routines.  Include order in the host
// translation unit:
//
//     #include "preprocessing/digasopre.h"      // the reference's structs
//     #include "preprocessing/preprocessing.cpp"
//     #define __SOLUTIONUPDATE                  // updateSol comes from here
//     #include "reference_shim.cpp"             // this file
//     #include "solvers/dgsolvers.cpp"          // unchanged
//
// and link libhfem_b200.so.  Routines replaced (reference file:line):
//   assembleLinearSystem  assembly/globalassembly.cpp:423-556
//   assembleRHS           assembly/globalassembly.cpp:559-616
//   computeResidualNorm   assembly/globalassembly.cpp:618-678
//   getQ                  assembly/elementassembly.cpp:1414-1479
//   updateSol             solvers/solutionupdate.cpp:70-98
//   computeOrdering, computePreconditioner, gmres   solvers/dgsolvers.cpp:16-20
//                         (closed archives; spec kernel/gmres_bilu0.m)
// Differences a caller sees: the face-block system (sys.Hg, sys.Rg) and the
// condensed element data (sol.DinvF, sol.DinvRu) stay in device memory, so
// those host vectors are not filled; sys.x receives the GMRES solution, and
// sol.UDG / sol.UH the updated state, as the reference's routines leave them.
// One problem per process (the context is created from the structs on the
// first call and kept).  A failing call reports through the reference's
// error() (print and exit), as the reference's routines do.
#include <cstdio>
#include <vector>

#include "../../include/hfem_b200.h"

namespace hfem_shim {

hfem_ctx* g_ctx = nullptr;
std::vector<double> g_rnorm_log;     // residual norm of every assembly, in call order
bool g_current = false;              // the device state is the one updateSol left in sol

inline void check(int rc, const char* what) {
    if (rc == 0) return;
    char msg[640];
    std::snprintf(msg, sizeof msg, "hfem_b200 %s failed (%d): %s\n", what, rc, g_ctx ? hfem_last_error(g_ctx) : "");
    error(msg);
}

// The context of this process's problem, created from the reference's structs.
inline hfem_ctx* context(sysstruct& sys, meshstruct& mesh, masterstruct& master, appstruct& app) {
    if (g_ctx) return g_ctx;
    const int nd = (int)app.nd, npv = (int)master.npv, npf = (int)master.npf[0], nfe = (int)master.nfe;
    hfem_dims d;
    d.nd = nd;
    d.npv = npv;
    d.npf = npf;
    d.nfe = nfe;
    d.ngv = (int)master.ngv;
    d.ngf = (int)master.ngf[0];
    d.ne = (int)mesh.ne;
    d.nf = (int)mesh.nf;
    d.nblocks = (int)sys.ent2ent.size();
    check(hfem_create(&d, 0, &g_ctx), "hfem_create");
    std::vector<int> perm((size_t)npf * nfe);
    for (int is = 0; is < nfe; is++)
        for (int k = 0; k < npf; k++) perm[(size_t)is * npf + k] = (int)master.perm[is][k];
    check(hfem_set_master(g_ctx, &master.shapvt[0], &master.shapvg[0], &master.shapvgdotshapvl[0],
                          &master.shapft[0][0], &master.shapfg[0][0], &master.shapfgdotshapfc[0][0], perm.data()),
          "hfem_set_master");
    std::vector<int> elcon(mesh.elcon.begin(), mesh.elcon.end()), t2f(mesh.t2f.begin(), mesh.t2f.end());
    std::vector<int> rs(sys.ent2entStart.begin(), sys.ent2entStart.end()), ci(sys.ent2ent.begin(), sys.ent2ent.end());
    check(hfem_set_mesh(g_ctx, &mesh.dgnodes[0], elcon.data(), t2f.data(), rs.data(), ci.data()), "hfem_set_mesh");
    bool bounded = false;
    for (size_t i = 0; i < mesh.bf.size(); i++) bounded = bounded || mesh.bf[i] < 0;
    if (bounded) {
        std::vector<int> bf(mesh.bf.begin(), mesh.bf.end()), bcm(app.bcm.begin(), app.bcm.end());
        check(hfem_set_boundary(g_ctx, bf.data(), (int)bcm.size(), bcm.data(), &app.bcs[0]), "hfem_set_boundary");
    }
    check(hfem_set_app(g_ctx, (int)app.appname), "hfem_set_app");
    check(hfem_set_models(g_ctx, (int)app.convStabMethod, (int)app.viscosityModel), "hfem_set_models");
    return g_ctx;
}

// Physics and state of the current call (the drivers change fc_u, fc_q, time
// and the source between calls).
inline void upload(hfem_ctx* c, solstruct& sol, appstruct& app, bool state = true) {
    check(hfem_set_physics(c, &app.physicsparam[0], (int)app.tdep, app.fc_u, app.fc_q, app.time), "hfem_set_physics");
    if (state)
        check(hfem_set_solution(c, &sol.UDG[0], &sol.UH[0], sol.SH.empty() ? nullptr : &sol.SH[0]),
              "hfem_set_solution");
    g_current = false;
}

}  // namespace hfem_shim

void assembleLinearSystem(sysstruct& sys, elemstruct* elems, meshstruct& mesh, masterstruct& master, solstruct& sol,
                          appstruct& app, tempstruct* temps) {
    hfem_ctx* c = hfem_shim::context(sys, mesh, master, app);
    hfem_shim::upload(c, sol, app);
    hfem_shim::check(hfem_assemble(c, &sol.rNorm), "hfem_assemble");
    hfem_shim::g_rnorm_log.push_back(sol.rNorm);
}

// The reference assembles the right-hand side alone when it reuses a Jacobian
// (quasi-Newton); the GPU assembly forms both at the same cost.
void assembleRHS(sysstruct& sys, elemstruct* elems, meshstruct& mesh, masterstruct& master, solstruct& sol,
                 appstruct& app, tempstruct* temps) {
    assembleLinearSystem(sys, elems, mesh, master, sol, app, temps);
}

void computeResidualNorm(sysstruct& sys, elemstruct* elems, meshstruct& mesh, masterstruct& master, solstruct& sol,
                         appstruct& app, tempstruct* temps) {
    // right after updateSol (the line search of solveNonlinearProblem) the
    // device already holds the state, together with the last solve's step,
    // which further updateSol calls still apply
    hfem_ctx* c = hfem_shim::context(sys, mesh, master, app);
    const bool current = hfem_shim::g_current;
    hfem_shim::upload(c, sol, app, !current);
    hfem_shim::check(hfem_residual(c, &sol.rNorm), "hfem_residual");
    hfem_shim::g_current = current;
}

// The reference's getQ works on one element; its callers (solveProblem and
// updateSol) loop over every element in order with sol's arrays.  The first
// element's call computes q for the whole mesh on the GPU and writes sol.UDG;
// the other calls find it done.
void getQ(elemstruct& elem, meshstruct& mesh, masterstruct& master, appstruct& app, solstruct& sol,
          tempstruct& temp, double* u, double* q, double* UH, double* sh, Int ie) {
    if (ie != 0) return;
    if (!hfem_shim::g_ctx)
        error("hfem_b200 getQ: call assembleLinearSystem or computeResidualNorm first (the GPU context is built "
              "from the solver structs)\n");
    hfem_shim::upload(hfem_shim::g_ctx, sol, app);
    hfem_shim::check(hfem_getq(hfem_shim::g_ctx), "hfem_getq");
    hfem_shim::check(hfem_get_solution(hfem_shim::g_ctx, &sol.UDG[0], nullptr), "hfem_get_solution");
}

// uh += alpha duh, u += alpha (D^-1 Ru - D^-1 F duh_e), q recomputed; duh is the
// solution of the last gmres call (sys.x), which is what the drivers pass.
void updateSol(sysstruct& sys, elemstruct* elems, meshstruct& mesh, masterstruct& master, solstruct& sol,
               appstruct& app, tempstruct* temps, Int* ndims, double* udg, double* uh, double* duh, double alpha) {
    hfem_shim::check(hfem_update(hfem_shim::g_ctx, alpha), "hfem_update");
    hfem_shim::check(hfem_get_solution(hfem_shim::g_ctx, udg, uh), "hfem_get_solution");
    hfem_shim::g_current = true;
}

// The ordering (minimum discarded fill for BILU0) is computed on the GPU by the
// next gmres call from the system it solves; this asks for a new one.
void computeOrdering(sysstruct& sys, Int preconditioner) {
    if (hfem_shim::g_ctx) hfem_shim::check(hfem_reset_ordering(hfem_shim::g_ctx), "hfem_reset_ordering");
}

// The preconditioner (0 BILU0, 2 block Jacobi, -1 none) is factored on the GPU
// by the gmres call that uses it.
void computePreconditioner(sysstruct& sys, Int preconditioner) {}

void gmres(sysstruct& sys, Int* convFlag) {
    int conv = 0, iters = 0;
    hfem_shim::check(hfem_gmres(hfem_shim::g_ctx, (int)sys.preconditioner, (int)sys.restart, sys.tol,
                                (int)sys.maxiter, &conv, &iters, nullptr, 0),
                     "hfem_gmres");
    *convFlag = conv;
    hfem_shim::check(hfem_download(hfem_shim::g_ctx, 7, &sys.x[0], sys.x.size()), "hfem_download");
}
