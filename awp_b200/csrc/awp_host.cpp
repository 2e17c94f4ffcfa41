// Host-side set-up: Q(f) tables, relaxation times, Cerjan sponge.
//
// Each routine restates one reference routine with the same float/double
// rounding points, so its output is bit-identical to the reference's
// (checked against the reference's own mesh.c / cerjan.c in the CPU tests).
#include "awp_host.h"

#include <math.h>

namespace awp {

namespace {

// Q(f) fitting tables of weights_sub (mesh.c:713-1097).  The data must be the
// reference's: they are the coefficients of its coarse-grained Q(f) fit.
// Weights are listed in the reference's order
//   [0][0][0] [1][0][0] [0][1][0] [1][1][0] [0][0][1] [1][0][1] [0][1][1] [1][1][1]
struct QBand {
  double lo, hi;  // lo <= EX < hi
  double w[8];
  double c[16];
};

const QBand kBands[] = {
    {0.01, 0.15,
     {0.3273, 1.0434, 0.044, 0.9393, 1.7268, 0.369, 0.8478, 0.4474},
     {7.3781, 4.1655, -83.1627, 13.1326, 69.0839, 0.4981, -37.6966, 5.5263,
      -51.4056, 8.1934, 13.1865, 3.4775, -36.1049, 7.2107, 12.3809, 3.6117}},
    {0.15, 0.25,
     {0.001, 1.0349, 0.0497, 1.0407, 1.7245, 0.2005, 0.804, 0.4452},
     {31.8902, 1.6126, -83.2611, 13.0749, 65.485, 0.5118, -42.02, 5.0875,
      -49.2656, 8.1552, 25.7345, 2.2801, -40.8942, 7.9311, 7.0206, 3.4692}},
    {0.25, 0.35,
     {0.001, 1.0135, 0.0621, 1.1003, 1.7198, 0.0918, 0.6143, 0.4659},
     {43.775, -0.1091, -83.1088, 13.0161, 60.9008, 0.592, -43.4857, 4.5869,
      -45.3315, 8.0252, 34.3571, 1.199, -41.4422, 8.399, -2.8772, 3.5323}},
    {0.35, 0.45,
     {0.001, 0.9782, 0.082, 1.1275, 1.7122, 0.001, 0.4639, 0.509},
     {41.6858, -0.7344, -164.2252, 14.9961, 103.0301, -0.4199, -41.1157, 3.8266,
      -73.0432, 8.5857, 38.0868, 0.3937, -43.2133, 8.6747, 5.6362, 3.3287}},
    {0.45, 0.55,
     {0.2073, 0.912, 0.1186, 1.081, 1.6984, 0.001, 0.1872, 0.6016},
     {20.0539, -0.4354, -81.6068, 12.8573, 45.9948, 1.1528, -23.07, 2.6719,
      -27.8961, 7.1927, 31.4788, -0.0434, -25.1661, 8.245, -45.2178, 4.8476}},
    {0.55, 0.65,
     {0.3112, 0.8339, 0.1616, 1.0117, 1.6821, 0.0001, 0.0001, 0.7123},
     {8.0848, -0.1968, -79.9715, 12.7318, 35.7155, 1.68, -13.0365, 1.8101,
      -13.2235, 6.3697, 25.4548, -0.3947, -10.4478, 7.657, -75.9179, 6.1791}},
    {0.65, 0.75,
     {0.1219, 0.001, 0.5084, 0.2999, 1.2197, 0.001, 0.001, 1.3635},
     {1.9975, 0.418, -76.6932, 11.3479, 40.7406, 1.9511, -2.7761, 0.5987, 0, 0,
      0, 0, 41.317, 2.1874, -88.8095, 11.0003}},
    {0.75, 0.85,
     {0.0462, 0.001, 0.4157, 0.1585, 1.3005, 0.001, 0.001, 1.4986},
     {5.1672, 0.2129, -46.506, 11.7213, -5.8873, 1.4279, -8.2448, 0.3455,
      15.0254, -0.283, 0, 0, 58.975, 0.8131, -108.6828, 12.4362}},
    {0.85, 0.95,
     {0.001, 0.001, 0.1342, 0.1935, 1.5755, 0.001, 0.001, 1.5297},
     {-0.8151, 0.1621, -61.9333, 12.5014, 0.0358, -0.0006, 0, 0, 22.0291,
      -0.4022, 0, 0, 56.0043, 0.7978, -116.9175, 13.0244}},
    {-1e300, 0.01,
     {0.8867, 1.0440, 0.0423, 0.8110, 1.7275, 0.5615, 0.8323, 0.4641},
     {-27.5089, 7.4177, -82.8803, 13.1952, 72.0312, 0.5298, -34.1779, 6.0293,
      -52.2607, 8.1754, -1.6270, 4.6858, -27.7770, 6.2852, 14.6295, 3.8839}},
};

// listing position -> flat index 4*i + 2*j + k
const int kListToFlat[8] = {0, 4, 2, 6, 1, 5, 3, 7};

}  // namespace

bool tau_range(float ex, float fac, float* taumax, float* taumin) {
  const float pi = 4. * atan(1.);
  const float twopi = 2 * pi;  // int * float, as in the reference
  *taumax = 1. / (twopi * 0.01) * 1.0 * fac;
  if (ex < 0.65 && ex >= 0.01) {
    *taumin = 1. / (twopi * 10.0) * 0.2 * fac;
  } else if (ex < 0.85 && ex >= 0.65) {
    *taumin = 1. / (twopi * 12.0) * 0.5 * fac;
    *taumax = 1. / (twopi * 0.08) * 2.0 * fac;
  } else if (ex < 0.95 && ex >= 0.85) {
    *taumin = 1. / (twopi * 15.0) * 0.8 * fac;
    *taumax = 1. / (twopi * 0.1) * 2.5 * fac;
  } else if (ex < 0.01) {
    *taumin = 1. / (twopi * 10.0) * 0.2 * fac;
  } else {
    return false;
  }
  return true;
}

void tausub(float taumin, float taumax, float tau8[8]) {
  // relaxation-time ordering of tausub, listed in the reference's order
  const float tautem[8] = {1.0f, 6.0f, 7.0f, 4.0f, 8.0f, 3.0f, 2.0f, 5.0f};
  const float prod = taumax * taumin;
  const float ratio = taumax / taumin;
  for (int n = 0; n < 8; ++n) {
    float tmp = tautem[n];
    tmp = (tmp - 0.5) / 8.0;
    tmp = 2.0 * tmp - 1.0;
    tau8[kListToFlat[n]] = exp(0.5 * (log((double)prod) + log((double)ratio) * tmp));
  }
}

bool weights_sub(float ex, float fac, float w8[8], float coeff16[16]) {
  const QBand* band = nullptr;
  for (const QBand& b : kBands)
    if (ex < b.hi && ex >= b.lo) {
      band = &b;
      break;
    }
  if (!band) {
    for (int n = 0; n < 8; ++n) w8[n] = 0.f;
    for (int n = 0; n < 16; ++n) coeff16[n] = 0.f;
    return false;
  }
  const double facex = pow((double)fac, (double)ex);
  for (int n = 0; n < 8; ++n) {
    const float w = (float)band->w[n];
    w8[kListToFlat[n]] = w / facex;
  }
  for (int n = 0; n < 16; ++n) coeff16[n] = (float)band->c[n];
  return true;
}

void texture_tables(const float tau8[8], const float w8[8], float dt, AwpTexture* t) {
  for (int n = 0; n < 8; ++n) {
    const float tauu = tau8[n];
    const float t2 = exp((double)(-dt / tauu));
    t->tau2[n] = t2;
    t->tau1[n] = 0.5 * (1. - t2);
    t->wwo8[n] = 8.0 * w8[n];
  }
}

void inicrj(float arbc, int nxt, int nyt, int nzt, int NX, int NY, int ND,
            int islowest, int npc, float* dcrjx, float* dcrjy, float* dcrjz) {
  (void)nzt;
  const float alpha = sqrt(-log((double)arbc)) / ND;
  int nxp = 1;  // nxt*coords[0] + 1 with coords = (0, 0)
  if (nxp <= ND && npc < 2) {
    for (int i = 0; i < ND; i++) {
      nxp = i + 1;
      dcrjx[i + 2 + AWP_NGSL] =
          dcrjx[i + 2 + AWP_NGSL] * (exp((double)-((alpha * (ND - nxp + 1)) * (alpha * (ND - nxp + 1)))));
    }
  }
  nxp = 1;
  if ((nxp + nxt - 1) >= (NX - ND + 1) && npc < 2) {
    for (int i = nxt - ND; i < nxt; i++) {
      nxp = i + NX - nxt + 1;
      dcrjx[i + 2 + AWP_NGSL] = dcrjx[i + 2 + AWP_NGSL] *
                                (exp((double)-((alpha * (ND - (NX - nxp))) * (alpha * (ND - (NX - nxp))))));
    }
  }
  int nyp = 1;
  if (nyp <= ND && npc < 2) {
    for (int j = 0; j < ND; j++) {
      nyp = j + 1;
      dcrjy[j + 2 + AWP_NGSL] =
          dcrjy[j + 2 + AWP_NGSL] * (exp((double)-((alpha * (ND - nyp + 1)) * (alpha * (ND - nyp + 1)))));
    }
  }
  nyp = 1;
  if ((nyp + nyt - 1) >= (NY - ND + 1) && npc < 2) {
    for (int j = nyt - ND; j < nyt; j++) {
      nyp = j + NY - nyt + 1;
      dcrjy[j + 2 + AWP_NGSL] = dcrjy[j + 2 + AWP_NGSL] *
                                (exp((double)-((alpha * (ND - (NY - nyp))) * ((alpha * (ND - (NY - nyp)))))));
    }
  }
  if (islowest) {
    for (int k = 0; k < ND; k++) {
      const int nzp = k + 1;
      dcrjz[k + AWP_ALIGN] =
          dcrjz[k + AWP_ALIGN] * (exp((double)-((alpha * (ND - nzp + 1)) * ((alpha * (ND - nzp + 1))))));
    }
  }
}

float qf_threshold() {
  float x = 0.005f;
  // step down while the smaller float still satisfies the switch
  for (;;) {
    const float y = nextafterf(x, 0.f);
    if (1.0 / (double)y <= 200.0) x = y; else break;
  }
  // step up until the switch holds
  while (!(1.0 / (double)x <= 200.0)) x = nextafterf(x, 1.f);
  return x;
}

void rotation_matrix(const float strike[3], const float dip[3], float Rz[9], float RzT[9]) {
  float alpha[3], beta[3];
  for (int k = 0; k < 3; k++) {
    alpha[k] = strike[k] / 180. * M_PI;
    beta[k] = dip[k] / 180. * M_PI;
  }
  Rz[0] = cosf(alpha[0]) * cosf(beta[0]);
  Rz[1] = sinf(alpha[0]) * cosf(beta[0]);
  Rz[2] = sinf(beta[0]);
  Rz[3] = cosf(alpha[1]) * cosf(beta[1]);
  Rz[4] = sinf(alpha[1]) * cosf(beta[1]);
  Rz[5] = sinf(beta[1]);
  Rz[6] = cosf(alpha[2]) * cosf(beta[2]);
  Rz[7] = sinf(alpha[2]) * cosf(beta[2]);
  Rz[8] = sinf(beta[2]);
  RzT[0] = Rz[0];
  RzT[1] = Rz[3];
  RzT[2] = Rz[6];
  RzT[3] = Rz[1];
  RzT[4] = Rz[4];
  RzT[5] = Rz[7];
  RzT[6] = Rz[2];
  RzT[7] = Rz[5];
  RzT[8] = Rz[8];
}

}  // namespace awp
