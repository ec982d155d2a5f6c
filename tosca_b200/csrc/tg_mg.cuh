// Geometric multigrid preconditioner of the pressure solve (see tg_mg.cu).
#pragma once

#include "tg_internal.cuh"

namespace tg {

struct MG;   // opaque; storage type chosen at creation (FP64 or FP32)

// face coefficients of the 7-point part of the fine operator on the compact
// interior grid (natural order c = (k*ny + j)*nx + i): aE/aN/aT of the
// east/north/top face of every cell, zero on non-periodic boundary faces
MG *mg_create(tg_ctx *C, bool fp32, const double *aE, const double *aN, const double *aT,
              int nx, int ny, int nz, int pi, int pj, int pk);
void mg_destroy(MG *mg);

// z = P M P^T r with P the shift that zeroes the pinned cell (natural index 0):
// the right-hand side at the pinned cell is replaced by -sum(r) (d_sum[0])
void mg_apply(tg_ctx *C, MG *mg, const double *r, const double *d_sum, double *z);

int mg_levels(const MG *mg);

}  // namespace tg
