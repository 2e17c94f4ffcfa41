// Host-side set-up shared by the context API and the pmcl3d driver.
#pragma once

#include "awp_common.h"

namespace awp {

// Relaxation-time range for the coarse-grained memory variables
// (inimesh, mesh.c:36-57).  Returns false for EX >= 0.95, where the reference
// leaves taumin unset.
bool tau_range(float ex, float fac, float* taumax, float* taumin);

// tausub (mesh.c:684-710): 8 relaxation times, index 4*ix + 2*iy + iz.
void tausub(float taumin, float taumax, float tau8[8]);

// weights_sub (mesh.c:713-1097): Q(f) weights (divided by FAC^EX) and the
// 16-entry coefficient table.  Returns false when EX lies outside every band.
bool weights_sub(float ex, float fac, float w8[8], float coeff16[16]);

// tau1/tau2 of pmcl3d.c:1036-1049 and the texture tables of init_texture.
void texture_tables(const float tau8[8], const float w8[8], float dt, AwpTexture* t);

// inicrj (cerjan.c:5-64) for a single rank (coords 0,0).
void inicrj(float arbc, int nxt, int nyt, int nzt, int NX, int NY, int ND,
            int islowest, int npc, float* dcrjx, float* dcrjy, float* dcrjz);

// Smallest float x > 0 with 1/(double)x <= 200.0 (the Q(f) branch switch of
// dstrqc, kernel.cu:974).
float qf_threshold();

// Rotation matrix of the principal-stress frame (mesh.c:1403-1431).
void rotation_matrix(const float strike[3], const float dip[3], float Rz[9], float RzT[9]);

}  // namespace awp
