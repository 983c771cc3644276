// Restatement of dmdserial, the face-to-face block CSR the reference builds in
// a closed archive (preprocessing/dmdserlib.a, called at
// preprocessing/preprocessing.cpp:14) -- TEST INFRASTRUCTURE ONLY.  Rows are
// faces, the diagonal block first (kernel/computeBILU0.m:15-17,
// kernel/mkBlockJacobi.m:10), then the other faces of the elements that share
// the row's face in increasing order.  Included after the reference headers.
#include <algorithm>
#include <set>
#include <vector>

void dmdserial(sysstruct& sys, meshstruct& mesh, appstruct& app)
{
    const Int nf = mesh.nf, ne = mesh.ne, nfe = mesh.nfemax;
    std::vector<std::set<Int> > rows(nf);
    for (Int e = 0; e < ne; e++)
        for (Int a = 0; a < nfe; a++)
            for (Int b = 0; b < nfe; b++)
                rows[mesh.t2f[e * nfe + a]].insert(mesh.t2f[e * nfe + b]);
    sys.ent2entStart.assign(nf + 1, 0);
    sys.ent2ent.clear();
    Int maxrow = 0;
    for (Int i = 0; i < nf; i++) {
        sys.ent2ent.push_back(i);
        for (Int j : rows[i]) if (j != i) sys.ent2ent.push_back(j);
        sys.ent2entStart[i + 1] = (Int)sys.ent2ent.size();
        maxrow = std::max(maxrow, sys.ent2entStart[i + 1] - sys.ent2entStart[i]);
    }
    sys.numEntities = nf;
    sys.numBlocks = (Int)sys.ent2ent.size();
    sys.blkSize = app.nch * mesh.npfmax;
    sys.maxBlocksPerRow = maxrow;
    sys.BJ_nrows = nf;
    sys.nproc = 1;
    sys.nentrecv = sys.nentsend = sys.nelemrecv = sys.nelemsend = 0;
    sys.nvecrecv = sys.nvecsend = sys.nmatrecv = sys.nmatsend = 0;
    sys.nnbsd = 0;
}
