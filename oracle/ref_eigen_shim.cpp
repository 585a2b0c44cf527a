// ref_eigen_shim.cpp -- C entry point over GARLI's own linalg.cpp, compiled from
// the reference sources by oracle/build_ref.sh into oracle/_ref/.  Test
// infrastructure only: it lets the CPU tests check the oracle's and the
// engine's eigensystems against Model::CalcEigenStuff's solver
// (EigenRealGeneral + InvertMatrix, model.cpp:827-856; linalg.cpp:95, :249).
#include <vector>
#include "defs.h"
#include "linalg.h"

extern "C" int ref_eigen(int n, const double *Q, double *eval, double *U, double *Uinv) {
    std::vector<double> a(n * n), u(n * n), ui(n * n), col(n), vi(n), work(n);
    std::vector<int> iwork(n), indx(n);
    std::vector<double *> ar(n), ur(n), uir(n);
    for (int i = 0; i < n; i++) {
        ar[i] = &a[i * n];
        ur[i] = &u[i * n];
        uir[i] = &ui[i * n];
    }
    for (int i = 0; i < n * n; i++) a[i] = Q[i];
    int rc = EigenRealGeneral(n, ar.data(), eval, vi.data(), ur.data(), iwork.data(), work.data());
    if (rc != 0) return rc;
    std::vector<double> t(u);
    std::vector<double *> tr(n);
    for (int i = 0; i < n; i++) tr[i] = &t[i * n];
    rc = InvertMatrix(tr.data(), n, col.data(), indx.data(), uir.data());
    for (int i = 0; i < n * n; i++) {
        U[i] = u[i];
        Uinv[i] = ui[i];
    }
    return rc;
}
