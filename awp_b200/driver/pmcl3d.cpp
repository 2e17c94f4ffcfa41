// pmcl3d -- single-rank drop-in for the reference's pmcl3d executable.
//
// Same command line (src/awp/command.c), same input files (INVEL mesh,
// INSRC sources or plane wave, sourcefilter.dat, nonlinear.dat, SOURCEFILE,
// RECVFILE, FORCEFILE and SGTFILE point sets, INTOPO topography) and the same output
// files (OUT/SX_0_%07ld, SY, SZ, Eta; the CHKFILE statistics log; the receiver
// files <file>_<x|y|z>_<step>; the SGT files <file>_<Gxx..Gyz>_<step> and the
// material files <file>_<d1|lami|mui>) as the reference's single-rank run; the
// time step itself runs in libawpb200 through its C ABI.
//
// Scope: one rank (PX = PY = 1, no I/O ranks), one grid or a discontinuous
// mesh of NGRIDS blocks (each 3x finer than the one below, pmcl3d.c:370-378),
// MEDIASTART 0-3, IFAULT 1, 2, 4, 5 and 6, NVE 1 and 3, FOLLOWBATHY 0 and 1.  On a
// mesh the SOURCEFILE / RECVFILE / FORCEFILE / SGTFILE point sets and the
// topography belong to the top block (grid 0).  Anything else is reported and
// refused.
#include <getopt.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/time.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/awp_b200.h"

#define MAXGRIDS 10
#define NGSL 8
#define ALIGN 32
#define NEDZ_EP 160

namespace {

struct Args {
  float TMAX = 20.00f, DH = 200.0f, DT = 0.01f, ARBC = 0.92f, PHT = 0.1f;
  int NPC = 0, ND = 20, NSRC[MAXGRIDS] = {1}, NST = 91, NVAR = 3, NVE = 1, MEDIASTART = 0;
  int IFAULT = 1, READ_STEP = 91, READ_STEP_GPU = 91, NTISKP = 1, WRITE_STEP = 10;
  int NX = 256, NY = 256, NZ[MAXGRIDS] = {1024}, PX = 1, PY = 1;
  int NBGX[MAXGRIDS], NEDX[MAXGRIDS], NSKPX[MAXGRIDS];
  int NBGY[MAXGRIDS], NEDY[MAXGRIDS], NSKPY[MAXGRIDS];
  int NBGZ[MAXGRIDS], NEDZ[MAXGRIDS], NSKPZ[MAXGRIDS];
  int IDYNA = 0, SoCalQ = 1;
  float FAC = 0.005f, Q0 = 5.0f, EX = 0.0f, FP = 2.5f;
  int NGRIDS = 1, FOLLOWBATHY = 0;
  std::string INSRC = "input/FAULTPOW", INVEL = "input/media", OUT = "output_sfc";
  std::string INSRC_I2 = "input_rst/srcpart/split_faults/fault", CHKFILE = "output_ckp/CHKP";
  std::string INTOPO = "input/topography", SOURCEFILE, RECVFILE, FORCEFILE, SGTFILE;
  int USETOPO = 0, USESOURCEFILE = 0, USERECVFILE = 0, USEFORCEFILE = 0, USESGTFILE = 0;
  Args() {
    for (int p = 0; p < MAXGRIDS; ++p) {
      NBGX[p] = NBGY[p] = NBGZ[p] = 1;
      NEDX[p] = NEDY[p] = -1;
      NEDZ[p] = 1;
      NSKPX[p] = NSKPY[p] = NSKPZ[p] = 1;
      if (p) NSRC[p] = 0, NZ[p] = 0;
    }
  }
};

void parsemultiple(const char* arg, int* val) {
  std::string s(arg);
  size_t pos = 0;
  int k = 0;
  while (k < MAXGRIDS) {
    size_t e = s.find(',', pos);
    val[k++] = atoi(s.substr(pos, e == std::string::npos ? std::string::npos : e - pos).c_str());
    if (e == std::string::npos) break;
    pos = e + 1;
  }
}

// command() of src/awp/command.c:152-546
void command(int argc, char** argv, Args& a) {
  static const char* optstring =
      "-T:H:t:A:P:M:D:S:N:V:B:n:I:R:Q:X:Y:Z:x:y:G:z:i:l:h:30:p:s:r:W:1:2:"
      "3:11:12:13:21:22:23:100:101:102:103:106:107:109:9:o:c:";
  static struct option long_options[] = {
      {"TMAX", required_argument, NULL, 'T'},     {"DH", required_argument, NULL, 'H'},
      {"DT", required_argument, NULL, 't'},       {"ARBC", required_argument, NULL, 'A'},
      {"PHT", required_argument, NULL, 'P'},      {"NPC", required_argument, NULL, 'M'},
      {"ND", required_argument, NULL, 'D'},       {"NSRC", required_argument, NULL, 'S'},
      {"NST", required_argument, NULL, 'N'},      {"NVE", required_argument, NULL, 'V'},
      {"MEDIASTART", required_argument, NULL, 'B'}, {"NVAR", required_argument, NULL, 'n'},
      {"IFAULT", required_argument, NULL, 'I'},   {"READ_STEP", required_argument, NULL, 'R'},
      {"READ_STEP_GPU", required_argument, NULL, 'Q'}, {"NX", required_argument, NULL, 'X'},
      {"NY", required_argument, NULL, 'Y'},       {"NZ", required_argument, NULL, 'Z'},
      {"PX", required_argument, NULL, 'x'},       {"PY", required_argument, NULL, 'y'},
      {"NGRIDS", required_argument, NULL, 'G'},   {"NBGX", required_argument, NULL, 1},
      {"NEDX", required_argument, NULL, 2},       {"NSKPX", required_argument, NULL, 3},
      {"NBGY", required_argument, NULL, 11},      {"NEDY", required_argument, NULL, 12},
      {"NSKPY", required_argument, NULL, 13},     {"NBGZ", required_argument, NULL, 21},
      {"NEDZ", required_argument, NULL, 22},      {"NSKPZ", required_argument, NULL, 23},
      {"IDYNA", required_argument, NULL, 'i'},    {"SoCalQ", required_argument, NULL, 's'},
      {"FAC", required_argument, NULL, 'l'},      {"Q0", required_argument, NULL, 'h'},
      {"EX", required_argument, NULL, 30},        {"FP", required_argument, NULL, 'p'},
      {"NTISKP", required_argument, NULL, 'r'},   {"WRITE_STEP", required_argument, NULL, 'W'},
      {"INSRC", required_argument, NULL, 100},    {"INVEL", required_argument, NULL, 101},
      {"OUT", required_argument, NULL, 'o'},      {"INSRC_I2", required_argument, NULL, 102},
      {"CHKFILE", required_argument, NULL, 'c'},  {"FOLLOWBATHY", required_argument, NULL, 7},
      {"INTOPO", required_argument, NULL, 103},   {"SOURCEFILE", required_argument, NULL, 107},
      {"RECVFILE", required_argument, NULL, 109}, {"FORCEFILE", required_argument, NULL, 9},
      {"SGTFILE", required_argument, NULL, 10},   {0, 0, 0, 0}};
  int insrcIsSet = 0, readstepGpuIsSet = 0, c;
  while ((c = getopt_long(argc, argv, optstring, long_options, NULL)) != -1) {
    switch (c) {
      case 'T': a.TMAX = atof(optarg); break;
      case 'H': a.DH = atof(optarg); break;
      case 't': a.DT = atof(optarg); break;
      case 'A': a.ARBC = atof(optarg); break;
      case 'P': a.PHT = atof(optarg); break;
      case 'M': a.NPC = atoi(optarg); break;
      case 'D': a.ND = atoi(optarg); break;
      case 'S': parsemultiple(optarg, a.NSRC); break;
      case 'N': a.NST = atoi(optarg); break;
      case 'V': a.NVE = atoi(optarg); break;
      case 'B': a.MEDIASTART = atoi(optarg); break;
      case 'n': a.NVAR = atoi(optarg); break;
      case 'I': a.IFAULT = atoi(optarg); break;
      case 'R': a.READ_STEP = atoi(optarg); break;
      case 'Q': readstepGpuIsSet = 1; a.READ_STEP_GPU = atoi(optarg); break;
      case 'X': a.NX = atoi(optarg); break;
      case 'Y': a.NY = atoi(optarg); break;
      case 'Z': parsemultiple(optarg, a.NZ); break;
      case 'x': a.PX = atoi(optarg); break;
      case 'y': a.PY = atoi(optarg); break;
      case 1: parsemultiple(optarg, a.NBGX); break;
      case 2: parsemultiple(optarg, a.NEDX); break;
      case 3: parsemultiple(optarg, a.NSKPX); break;
      case 11: parsemultiple(optarg, a.NBGY); break;
      case 12: parsemultiple(optarg, a.NEDY); break;
      case 13: parsemultiple(optarg, a.NSKPY); break;
      case 21: parsemultiple(optarg, a.NBGZ); break;
      case 22: parsemultiple(optarg, a.NEDZ); break;
      case 23: parsemultiple(optarg, a.NSKPZ); break;
      case 'i': a.IDYNA = atoi(optarg); break;
      case 's': a.SoCalQ = atoi(optarg); break;
      case 'l': a.FAC = atof(optarg); break;
      case 'h': a.Q0 = atof(optarg); break;
      case 30: a.EX = atof(optarg); break;
      case 'p': a.FP = atof(optarg); break;
      case 'r': a.NTISKP = atoi(optarg); break;
      case 'W': a.WRITE_STEP = atoi(optarg); break;
      case 100: insrcIsSet = 1; a.INSRC = optarg; break;
      case 101: a.INVEL = optarg; break;
      case 'o': a.OUT = optarg; break;
      case 102: a.INSRC_I2 = optarg; break;
      case 'c': a.CHKFILE = optarg; break;
      case 'G': a.NGRIDS = atoi(optarg); break;
      case 7: a.FOLLOWBATHY = atoi(optarg); break;
      case 103: a.INTOPO = optarg; a.USETOPO = 1; break;
      case 107: a.SOURCEFILE = optarg; a.USESOURCEFILE = 1; break;
      case 109: a.RECVFILE = optarg; a.USERECVFILE = 1; break;
      case 9: a.FORCEFILE = optarg; a.USEFORCEFILE = 1; break;
      case 10: a.SGTFILE = optarg; a.USESGTFILE = 1; break;
      default:
        printf("Usage: %s \nOptions:\n\t[(-T | --TMAX) <TMAX>]\n\t[(-H | --DH) <DH>]\n"
               "\t[(-t | --DT) <DT>]\n\t[(-A | --ARBC) <ARBC>]\n\t[(-P | --PHT) <PHT>]\n"
               "\t[(-M | --NPC) <NPC>]\n\t[(-D | --ND) <ND>]\n\t[(-S | --NSRC) <NSRC>]\n"
               "\t[(-N | --NST) <NST>]\n",
               argv[0]);
        exit(-1);
    }
  }
  if (a.IFAULT == 2 && !insrcIsSet) a.INSRC = "input_rst/srcpart/tpsrc/tpsrc";
  if (!readstepGpuIsSet) a.READ_STEP_GPU = a.READ_STEP;
  if (a.NBGX[0] == 0) a.NBGX[0] = 1;
}

// calcRecordingPoints (src/awp/calc.c:9-72) at coords (0, 0)
void calc_recording_points(int* nbgx, int* nedx, int* nbgy, int* nedy, int* nbgz, int* nedz,
                           int* rnx, int* rny, int* rnz, long nxt, long nyt, long nzt, int NBGX,
                           int NEDX, int NSKPX, int NBGY, int NEDY, int NSKPY, int NBGZ, int NEDZ,
                           int NSKPZ) {
  *nbgx = *nedx = *nbgy = *nedy = *nbgz = *nedz = 0;
  if (NBGX > nxt) *rnx = 0;
  else if (NEDX < 1) *rnx = 0;
  else {
    *nbgx = NBGX - 1;
    *nedx = (nxt <= NEDX) ? (int)((nxt + NBGX - 1) % NSKPX - NSKPX + nxt) : NEDX - 1;
    *rnx = (*nedx - *nbgx) / NSKPX + 1;
  }
  if (NBGY > nyt) *rny = 0;
  else if (NEDY < 1) *rny = 0;
  else {
    *nbgy = NBGY - 1;
    *nedy = (nyt <= NEDY) ? (int)((nyt + NBGY - 1) % NSKPY - NSKPY + nyt) : NEDY - 1;
    *rny = (*nedy - *nbgy) / NSKPY + 1;
  }
  if (NBGZ > nzt) *rnz = 0;
  else {
    *nbgz = NBGZ - 1;
    *nedz = NEDZ - 1;
    *rnz = (*nedz - *nbgz) / NSKPZ + 1;
  }
  if (*rnx == 0 || *rny == 0 || *rnz == 0) {
    *rnx = *rny = *rnz = 0;
    *nedx = *nbgx - 1;
    *nedy = *nbgy - 1;
  }
}

double now() {
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

void die(const char* what, int st) {
  fprintf(stderr, "pmcl3d: %s failed: %s (%s)\n", what, awp_status_string(st), awp_last_error());
  exit(1);
}
#define AWP(call)                  \
  do {                             \
    int st_ = (call);              \
    if (st_) die(#call, st_);      \
  } while (0)

// IFAULT 4: frames of a previous run's volume output, the sub-volume of
// read_awp_subvolume (source.c:377-461) -- frame t of a file is nx*ny*nz
// floats; the rows of x0..x1-1 at every (k, j), k from the bottom of the file
// up with SEISM-IO output, else the file's k = nz-1-k walked from k1-1 down
// to k0 -- in the order of the points of read_src_ifault_4.
struct FrameFiles {
  std::string name[3];
  int dim[3];
  int ext[6];  // global half-open extents x0 x1 y0 y1 z0 z1 in the files
  int seismio;
};

int read_frames(void* user, int first, int n, float* vx, float* vy, float* vz) {
  const FrameFiles& F = *(const FrameFiles*)user;
  float* out[3] = {vx, vy, vz};
  const long long nx = F.dim[0], ny = F.dim[1], nz = F.dim[2], nel = nx * ny * nz;
  const int x0 = F.ext[0], x1 = F.ext[1], y0 = F.ext[2], y1 = F.ext[3], z0 = F.ext[4],
            z1 = F.ext[5];
  const int nx1 = x1 - x0;
  for (int q = 0; q < 3; ++q) {
    FILE* f = fopen(F.name[q].c_str(), "rb");
    if (!f) {
      fprintf(stderr, "pmcl3d: cannot open %s\n", F.name[q].c_str());
      return 1;
    }
    float* o = out[q];
    for (int t = first; t < first + n; ++t)
      for (int kk = 0; kk < z1 - z0; ++kk) {
        const long long kp = F.seismio ? (long long)(z0 + kk) : nz - (z1 - 1 - kk) - 1;
        for (int j = y0; j < y1; ++j) {
          const long long at = (long long)t * nel + kp * nx * ny + (long long)j * nx + x0;
          if (fseeko(f, (off_t)(at * (long long)sizeof(float)), SEEK_SET) ||
              fread(o, sizeof(float), nx1, f) != (size_t)nx1) {
            fclose(f);
            fprintf(stderr, "pmcl3d: %s: frame %d outside the file\n", F.name[q].c_str(), t);
            return 2;
          }
          o += nx1;
        }
      }
    fclose(f);
  }
  return 0;
}

// hoek_brown (mesh.c:1139-1176)
void hoek_brown(float sigma_0, float sigma_ci, float GSI, float mi, float D, int tunnel,
                float* phi, float* cohes) {
  double mb, s, a, sigma_cm, sigma_3max, sigma_3n, tmp;
  mb = (double)mi * exp(((double)GSI - 100.) / (28. - 14. * D));
  s = exp(((double)GSI - 100.) / (9. - 3. * (double)D));
  a = 1. / 2. + 1. / 6. * (exp(-(double)GSI / 15.) - exp(-20. / 3.));
  sigma_cm = (double)sigma_ci * (mb + 4. * s - a * (mb - 8. * s)) * pow(mb / 4. + s, a - 1.) /
             (2. * (1. + a) * (2. + a));
  if (tunnel == 0)
    sigma_3max = sigma_cm * 0.72 * pow(sigma_cm / sigma_0, -0.91);
  else
    sigma_3max = sigma_cm * 0.47 * pow(sigma_cm / sigma_0, -0.94);
  sigma_3n = sigma_3max / sigma_ci;
  tmp = 6. * a * mb * pow(s + mb * sigma_3n, a - 1.) /
        (2. * (1. + a) * (2. + a) + 6 * a * mb * pow(s + mb * sigma_3n, a - 1.));
  const double phi2 = asin(tmp) / M_PI * 180.;
  const double cohes2 = (sigma_ci * ((1. + 2 * a) * s + (1. - a) * mb * sigma_3n) *
                         pow(s + mb * sigma_3n, a - 1.)) /
                        ((1. + a) * (2. + a) *
                         sqrt(1. + (6 * a * mb * pow(s + mb * sigma_3n, a - 1.)) /
                                       ((1. + a) * (2. + a))));
  *phi = (float)phi2;
  *cohes = (float)cohes2;
}

}  // namespace

int main(int argc, char** argv) {
  Args A;
  command(argc, argv, A);
  double time_init = now();
  if (A.PX != 1 || A.PY != 1) {
    fprintf(stderr, "pmcl3d: this build runs one rank (PX = PY = 1)\n");
    return 1;
  }
  const int G = A.NGRIDS;
  if (G < 1 || G > MAXGRIDS) {
    fprintf(stderr, "pmcl3d: NGRIDS=%d is outside 1..%d\n", G, MAXGRIDS);
    return 1;
  }
  // block sizes of the mesh (pmcl3d.c:370-378): NX, NY, DH are the coarsest
  // block's, each block above is 3x finer
  int grdfct[MAXGRIDS], nxt[MAXGRIDS], nyt[MAXGRIDS], nzt[MAXGRIDS];
  float DHp[MAXGRIDS];
  grdfct[G - 1] = 1;
  for (int p = G - 2; p >= 0; --p) grdfct[p] = grdfct[p + 1] * 3;
  for (int p = 0; p < G; ++p) {
    DHp[p] = A.DH / grdfct[p];
    nxt[p] = A.NX * grdfct[p];
    nyt[p] = A.NY * grdfct[p];
    nzt[p] = A.NZ[p];
    if (nzt[p] % 4 != 0) {  // pmcl3d.c:380-391 (BLOCK_SIZE_Z = 4)
      fprintf(stderr,
              "NZT for grid %d is not divisble by BLOCK_SIZE_Z.\nNZT = %d, BLOCK_SIZE_Z=4\n", p,
              nzt[p]);
      return 0;
    }
  }
  const long nt = (int)(A.TMAX / A.DT) + 1;

  // recording points (pmcl3d.c:425-471)
  int grid_output[MAXGRIDS] = {0}, recNX[MAXGRIDS], recNY[MAXGRIDS], recNZ[MAXGRIDS];
  int rnbgx[MAXGRIDS], rnedx[MAXGRIDS], rnbgy[MAXGRIDS], rnedy[MAXGRIDS], rnbgz[MAXGRIDS],
      rnedz[MAXGRIDS], rnx[MAXGRIDS], rny[MAXGRIDS], rnz[MAXGRIDS];
  for (int p = 0; p < G; ++p) {
    if (p == 0) {
      if (A.NEDX[p] == -1) A.NEDX[p] = A.NX * grdfct[p];
      if (A.NEDY[p] == -1) A.NEDY[p] = A.NY * grdfct[p];
      if (A.NEDZ[p] == -1) A.NEDZ[p] = A.NZ[p];
      grid_output[p] = 1;
    }
    A.NEDX[p] = A.NEDX[p] - (A.NEDX[p] - A.NBGX[p]) % A.NSKPX[p];
    A.NEDY[p] = A.NEDY[p] - (A.NEDY[p] - A.NBGY[p]) % A.NSKPY[p];
    A.NEDZ[p] = A.NEDZ[p] - (A.NEDZ[p] - A.NBGZ[p]) % A.NSKPZ[p];
    if (A.NEDX[p] > -1 && A.NEDY[p] > -1 && A.NEDZ[p] > -1) grid_output[p] = 1;
    recNX[p] = (A.NEDX[p] - A.NBGX[p]) / A.NSKPX[p] + 1;
    recNY[p] = (A.NEDY[p] - A.NBGY[p]) / A.NSKPY[p] + 1;
    recNZ[p] = (A.NEDZ[p] - A.NBGZ[p]) / A.NSKPZ[p] + 1;
    calc_recording_points(&rnbgx[p], &rnedx[p], &rnbgy[p], &rnedy[p], &rnbgz[p], &rnedz[p],
                          &rnx[p], &rny[p], &rnz[p], nxt[p], nyt[p], nzt[p], A.NBGX[p],
                          A.NEDX[p], A.NSKPX[p], A.NBGY[p], A.NEDY[p], A.NSKPY[p], A.NBGZ[p],
                          A.NEDZ[p], A.NSKPZ[p]);
    if (!grid_output[p]) rnx[p] = rny[p] = rnz[p] = 0;
  }

  if (A.IFAULT != 1 && A.IFAULT != 2 && A.IFAULT != 4 && A.IFAULT != 5 && A.IFAULT != 6) {
    fprintf(stderr, "pmcl3d: IFAULT=%d sources are not part of this build\n", A.IFAULT);
    return 1;
  }
  if (A.IFAULT == 6) {  // pmcl3d.c:751-761
    printf("Using plane wave input at grid position %d in grid %d\n", A.NZ[G - 1] - A.ND - 1,
           G - 1);
    if (A.READ_STEP != A.NST) {
      fprintf(stderr, "Error.  READ_STEP should be equal NST for IFAULT=6\n");
      return 1;
    }
    if (A.NST < 1) {
      fprintf(stderr, "Error.  NST=%d, but should be > 0 for IFAULT=6.\n", A.NST);
      return 1;
    }
  }
  if (A.IFAULT == 5 && (A.NST != 2 || A.READ_STEP != 2)) {  // pmcl3d.c:680-688
    fprintf(stderr, "IFAULT=5 requires NST = READ_STEP =2.\nQuitting.");
    return -1;
  }
  awp_params P[MAXGRIDS];
  for (int p = 0; p < G; ++p) {
    awp_params_default(&P[p]);
    P[p].nx = nxt[p]; P[p].ny = nyt[p]; P[p].nz = nzt[p];
    P[p].dh = DHp[p]; P[p].dt = A.DT; P[p].arbc = A.ARBC; P[p].npc = A.NPC;
    P[p].nd = A.ND * grdfct[p];  // inicrj with ND*grdfct[p] (pmcl3d.c:1029)
    P[p].nve = (A.NVE == 3) ? 3 : 1;
    P[p].fac = A.FAC; P[p].q0 = A.Q0; P[p].ex = A.EX; P[p].fp = A.FP; P[p].socalq = A.SoCalQ;
    // IFAULT 2 windows of READ_STEP samples are assembled here into all NST
    P[p].ifault = A.IFAULT; P[p].nst = A.NST;
    P[p].read_step = (A.IFAULT == 2) ? std::max(A.NST, 1) : A.READ_STEP_GPU;
    P[p].grid = p;
    P[p].ngrids = G;
  }
  awp_mesh* mesh = nullptr;
  awp_ctx* ctx[MAXGRIDS] = {};
  if (G == 1) {
    AWP(awp_ctx_create(&P[0], &ctx[0]));
  } else {
    AWP(awp_mesh_create(P, G, &mesh));
    for (int p = 0; p < G; ++p) AWP(awp_mesh_grid(mesh, p, &ctx[p]));
  }

  // ---- sources (inisource, source.c:131-264; sourcefilter.dat, pmcl3d.c:651-675)
  int filtorder = 0;
  double fb[20] = {0}, fa[20] = {0};
  if (access("sourcefilter.dat", F_OK) != -1) {
    FILE* f = fopen("sourcefilter.dat", "r");
    if (fscanf(f, "%d\n", &filtorder) != 1) filtorder = 0;
    printf("Order of source filter: %d.  Parameters:\n", filtorder);
    for (int k = 0; k < filtorder + 1 && k < 20; k++) {
      if (fscanf(f, "%le %le\n", fb + k, fa + k) != 2) break;
      printf("b[%d]=%le, a[%d]=%le\n", k, fb[k], k, fa[k]);
    }
    fclose(f);
    for (int p = 0; p < G; ++p) AWP(awp_set_source_filter(ctx[p], filtorder, fb, fa));
  }
  std::vector<int> spos[MAXGRIDS];
  int nsrc[MAXGRIDS] = {0};
  for (int p = 0; p < G; ++p) {  // INSRC_<p> for every block with sources (pmcl3d.c:702-708)
    if (A.NSRC[p] <= 0 || !(A.IFAULT < 3 || A.IFAULT == 5)) continue;
    if (A.IFAULT == 2) {
      // read_src_ifault_2 (source.c:15-128) at rank 0: the header
      // "<INSRC>_<p>0000000" (npsrc, two words, positions), then the READ_STEP
      // windows "<INSRC_I2>_<p>0000000_<idx>", idx from 1, of six component
      // arrays (xx yy zz xz yz xy), each time-major with the sources fastest;
      // the time loop reads window idx at step (idx-1)*READ_STEP
      // (pmcl3d.c:2442-2461) while it is below NST
      char name[600];
      snprintf(name, sizeof(name), "%s_%d%07d", A.INSRC.c_str(), p, 0);
      FILE* f = fopen(name, "rb");
      if (!f) continue;  // no sources in this partition
      printf("SOURCE reading first time: %s\n", name);
      int np = 0, dummy[2];
      if (fread(&np, sizeof(int), 1, f) != 1 || fread(dummy, sizeof(int), 2, f) != 2 || np < 0) {
        fclose(f);
        fprintf(stderr, "pmcl3d: %s: bad header\n", name);
        return 1;
      }
      std::vector<int> pos((size_t)np * 3);
      if (fread(pos.data(), sizeof(int), pos.size(), f) != pos.size()) {
        fclose(f);
        fprintf(stderr, "pmcl3d: %s: %d positions expected\n", name, np);
        return 1;
      }
      fclose(f);
      if (np == 0) continue;
      const int RS = A.READ_STEP, N = std::max(A.NST, 1);
      if (RS < 1) {
        fprintf(stderr, "pmcl3d: IFAULT=2 needs READ_STEP >= 1\n");
        return 1;
      }
      std::vector<float> sdat((size_t)np * N * 6, 0.f), win((size_t)np * RS);
      for (int idx = 1; (long)(idx - 1) * RS < N; ++idx) {
        snprintf(name, sizeof(name), "%s_%d%07d_%03d", A.INSRC_I2.c_str(), p, 0, idx);
        printf("SOURCE reading: %s\n", name);
        FILE* g = fopen(name, "rb");
        if (!g) {
          printf("ERROR! Rank=%d: Cannot open file: %s\n", 0, name);
          return 1;
        }
        for (int q = 0; q < 6; ++q) {
          if (fread(win.data(), sizeof(float), win.size(), g) != win.size()) {
            fclose(g);
            fprintf(stderr, "pmcl3d: %s: short window\n", name);
            return 1;
          }
          for (int t = 0; t < RS; ++t) {
            const long step = (long)(idx - 1) * RS + t;
            if (step >= N) break;
            for (int s = 0; s < np; ++s)
              sdat[((size_t)s * N + step) * 6 + q] = win[(size_t)t * np + s];
          }
        }
        fclose(g);
      }
      nsrc[p] = np;
      spos[p] = pos;
      AWP(awp_upload_sources(ctx[p], np, pos.data(), sdat.data()));
      continue;
    }
    char name[512];
    snprintf(name, sizeof(name), "%s_%d", A.INSRC.c_str(), p);
    FILE* f = fopen(name, "rb");
    if (!f) {
      printf("can't open file %s", name);
      continue;
    }
    std::vector<float> tmp((size_t)A.NST * 6), sdat;
    const int rs = A.READ_STEP_GPU;
    for (int i = 0; i < A.NSRC[p]; ++i) {
      int t3[3];
      if (fread(t3, sizeof(int), 3, f) != 3 ||
          fread(tmp.data(), sizeof(float), tmp.size(), f) != tmp.size())
        break;
      spos[p].insert(spos[p].end(), t3, t3 + 3);
      for (int j = 0; j < rs; ++j)
        for (int q = 0; q < 6; ++q) sdat.push_back(j < A.NST ? tmp[(size_t)j * 6 + q] : 0.f);
      ++nsrc[p];
    }
    fclose(f);
    if (nsrc[p]) AWP(awp_upload_sources(ctx[p], nsrc[p], spos[p].data(), sdat.data()));
  }
  static FrameFiles frames;  // read by the library at every window
  if (A.IFAULT == 4) {
    // read_src_ifault_4 (source.c:469-680) at rank 0: the INSRC text gives the
    // x, y, z extents of the prescribed volume, the dimensions of the previous
    // run's output, the offset of this grid in it, the file mask (%c = X, Y,
    // Z), the SEISM-IO flag and the output step of that run
    FILE* f = fopen(A.INSRC.c_str(), "r");
    if (!f) {
      perror("could not open INSRC file");
      return 1;
    }
    int ext[6] = {0}, dim[3] = {0}, off[3] = {0}, seismio = 0, tskp = 1;
    char line[1024], mask[512] = "";
    int got = 0;
    if (fgets(line, sizeof line, f)) got += sscanf(line, "%d %d", ext, ext + 1);
    if (fgets(line, sizeof line, f)) got += sscanf(line, "%d %d", ext + 2, ext + 3);
    if (fgets(line, sizeof line, f)) got += sscanf(line, "%d %d", ext + 4, ext + 5);
    if (fgets(line, sizeof line, f)) got += sscanf(line, "%d %d %d", dim, dim + 1, dim + 2);
    if (fgets(line, sizeof line, f)) got += sscanf(line, "%d %d %d", off, off + 1, off + 2);
    if (fgets(line, sizeof line, f)) got += sscanf(line, "%511s", mask);
    if (fgets(line, sizeof line, f)) got += sscanf(line, "%d", &seismio);
    if (fgets(line, sizeof line, f)) got += sscanf(line, "%d", &tskp);
    fclose(f);
    if (got != 15) {
      fprintf(stderr, "pmcl3d: %s: eight lines of IFAULT=4 parameters expected\n",
              A.INSRC.c_str());
      return 1;
    }
    printf("fbc_pmask=\"%s\"\nfbc_seismio=%d\nfbc_tskp=%d\n", mask, seismio, tskp);
    // one rank: nbx = nby = 1 - 2*loop = -1, so the local extents are the
    // file's, clipped to the grid and its ghost cells
    const int westm = 1 - NGSL, eastm = nxt[0] + NGSL, southm = 1 - NGSL, northm = nyt[0] + NGSL;
    int extl[6] = {std::max(ext[0], westm), std::min(ext[1], eastm), std::max(ext[2], southm),
                   std::min(ext[3], northm), ext[4], ext[5]};
    long long npsrc = -1;
    if (extl[0] < eastm && extl[1] > westm && extl[2] < northm && extl[3] > southm)
      npsrc = (long long)(extl[1] - extl[0] + 1) * (extl[3] - extl[2] + 1) *
              (extl[5] - extl[4] + 1);
    printf("(0) npsrc=%lld\n", npsrc);
    if (npsrc > 0) {
      std::vector<int> pos;
      pos.reserve((size_t)npsrc * 3);
      for (int kk = 0; kk <= extl[5] - extl[4]; ++kk) {
        const int k = seismio ? extl[5] - kk : extl[4] + kk;
        for (int j = extl[2]; j <= extl[3]; ++j)
          for (int i = extl[0]; i <= extl[1]; ++i) {
            pos.push_back(i);
            pos.push_back(j);
            pos.push_back(nzt[0] - k + 1);
          }
      }
      // background_velocity_reader (source.c:684-793): global extents
      frames.ext[0] = extl[0] + off[0] - 1; frames.ext[1] = extl[1] + off[0];
      frames.ext[2] = extl[2] + off[1] - 1; frames.ext[3] = extl[3] + off[1];
      frames.ext[4] = extl[4] + off[2] - 1; frames.ext[5] = extl[5] + off[2];
      // the mask names the component with %c (sprintf(xfile, fbc_pmask, 'X'))
      const std::string m = mask;
      const size_t at = m.find("%c");
      if (at == std::string::npos || m.find('%', at + 2) != std::string::npos ||
          m.find('%') != at) {
        fprintf(stderr, "pmcl3d: %s: the file mask must hold one %%c\n", mask);
        return 1;
      }
      for (int q = 0; q < 3; ++q) {
        frames.name[q] = m.substr(0, at) + "XYZ"[q] + m.substr(at + 2);
        frames.dim[q] = dim[q];
      }
      frames.seismio = seismio;
      AWP(awp_velocity_forcing_init(ctx[0], (int)npsrc, pos.data(), A.NST, tskp,
                                    A.READ_STEP_GPU, read_frames, &frames));
    }
  }
  if (A.IFAULT == 5) printf("Using IFAULT=5: kinematic source.\n");
  if (A.IFAULT == 6) {  // ini_plane_wave (source.c:797-833): NST lines "vx vy vz"
    std::vector<float> pv[3];
    FILE* f = fopen(A.INSRC.c_str(), "r");
    if (!f) {
      perror(("Could not open " + A.INSRC).c_str());
      return 1;
    }
    for (int i = 0; i < A.NST; ++i) {
      float v[3];
      if (fscanf(f, "%e %e %e\n", v, v + 1, v + 2) < 3) {
        fprintf(stderr, "pmcl3d: %s holds fewer than NST=%d samples\n", A.INSRC.c_str(),
                A.NST);
        fclose(f);
        return 1;
      }
      for (int q = 0; q < 3; ++q) pv[q].push_back(v[q]);
    }
    fclose(f);
    AWP(awp_upload_plane_wave(ctx[G - 1], A.NST, pv[0].data(), pv[1].data(), pv[2].data()));
  }

  // ---- media (inimesh, mesh.c:23-614), INVEL_<p> per block (pmcl3d.c:882-892) ---
  float vse[MAXGRIDS][2] = {}, vpe[MAXGRIDS][2] = {}, dde[MAXGRIDS][2] = {};
  size_t ncell[MAXGRIDS];
  long long dims[MAXGRIDS][3];
  for (int p = 0; p < G; ++p) {
    AWP(awp_padded_dims(ctx[p], dims[p]));
    ncell[p] = (size_t)dims[p][0] * dims[p][1] * dims[p][2];
    if (A.MEDIASTART == 0) {
      float vp, vs, dd;
      if (A.IDYNA == 1) vp = 6000.0, vs = 3464.0, dd = 2670.0;
      else vp = 1500.0, vs = 500.0, dd = 2000.0;
      std::vector<float> lam(ncell[p], (float)(1. / (dd * (vp * vp - 2. * vs * vs)))),
          mu(ncell[p], (float)(1. / (dd * vs * vs))), d1(ncell[p], dd);
      AWP(awp_field_upload(ctx[p], AWP_D1, d1.data()));
      AWP(awp_field_upload(ctx[p], AWP_MU, mu.data()));
      AWP(awp_field_upload(ctx[p], AWP_LAM, lam.data()));
      vse[p][0] = vse[p][1] = vs; vpe[p][0] = vpe[p][1] = vp; dde[p][0] = dde[p][1] = dd;
    } else if (A.MEDIASTART >= 1 && A.MEDIASTART <= 3) {
      char name[512];
      if (A.MEDIASTART < 3) {
        snprintf(name, sizeof(name), "%s_%d", A.INVEL.c_str(), p);
      } else {  // the partition of rank 0 (mesh.c:138-141), the same name for every block
        snprintf(name, sizeof(name), "input_rst/mediapart/media%07d.bin", 0);
        printf("Rank=%d, reading file=%s\n", 0, name);
      }
      const size_t n = (size_t)A.NVAR * nxt[p] * nyt[p] * nzt[p];
      std::vector<float> m(n);
      FILE* f = fopen(name, "rb");
      if (!f || fread(m.data(), sizeof(float), n, f) != n) {
        printf("can't open file %s", name);
        return 1;
      }
      fclose(f);
      AWP(awp_upload_media(ctx[p], A.NVAR, m.data()));
      AWP(awp_media_extrema(ctx[p], vse[p], vpe[p], dde[p]));
    } else {
      fprintf(stderr, "pmcl3d: MEDIASTART=%d is not part of this build\n", A.MEDIASTART);
      return 1;
    }
  }

  // ---- FOLLOWBATHY surface levels of grid 0 (pmcl3d.c:905-930) ---------------
  if (A.FOLLOWBATHY == 1) {
    const long long nxp = dims[0][0], nyp = dims[0][1];
    std::vector<int> bathy((size_t)(nxp * nyp));
    AWP(awp_compute_bathymetry(ctx[0], bathy.data()));
    std::vector<float> mu(ncell[0]), d1(ncell[0]);
    AWP(awp_field_download(ctx[0], AWP_MU, mu.data()));
    AWP(awp_field_download(ctx[0], AWP_D1, d1.data()));
    mkdir("debug", 0755);
    FILE* fb = fopen("debug/bathy.0000", "w");
    if (fb) {
      for (long long i = 0; i < nxp; ++i)
        for (long long j = 0; j < nyp; ++j) {
          const int k = bathy[(size_t)(j * nxp + i)];
          if (k == 0) continue;
          const size_t q = (size_t)((i * nyp + j) * dims[0][2] + k);
          const float tmpvs = (float)sqrt(1. / (mu[q] * d1[q]));
          fprintf(fb, "%lld %lld %d %e\n", i, j, k, tmpvs);
        }
      fclose(fb);
    }
    AWP(awp_set_bathymetry(ctx[0], bathy.data()));
  }

  // ---- CHK statistics file (writeCHK, io.c:9-43) -----------------------------
  FILE* fchk = fopen(A.CHKFILE.c_str(), "w");
  if (fchk) {
    for (int p = 0; p < G; ++p) {
      fprintf(fchk, "-------------------------------------------------------------\n");
      fprintf(fchk, "GRID NUMBER:\t%d\n", p);
      fprintf(fchk, "STABILITY CRITERIA .5 > CMAX*DT/DX:\t%f\n", vpe[p][1] * A.DT / DHp[p]);
      fprintf(fchk, "# OF X,Y,Z NODES PER PROC:\t%d, %d, %d\n", nxt[p], nyt[p], nzt[p]);
      fprintf(fchk, "DISCRETIZATION IN SPACE:\t%f\n", DHp[p]);
      fprintf(fchk, "HIGHEST P-VELOCITY ENCOUNTERED:\t%f\n", vpe[p][1]);
      fprintf(fchk, "LOWEST P-VELOCITY ENCOUNTERED:\t%f\n", vpe[p][0]);
      fprintf(fchk, "HIGHEST S-VELOCITY ENCOUNTERED:\t%f\n", vse[p][1]);
      fprintf(fchk, "LOWEST S-VELOCITY ENCOUNTERED:\t%f\n", vse[p][0]);
      fprintf(fchk, "HIGHEST DENSITY ENCOUNTERED:\t%f\n", dde[p][1]);
      fprintf(fchk, "LOWEST  DENSITY ENCOUNTERED:\t%f\n", dde[p][0]);
      fprintf(fchk, "-------------------------------------------------------------\n");
    }
    fprintf(fchk, "# OF TIME STEPS:\t%ld\n", nt);
    fprintf(fchk, "DISCRETIZATION IN TIME:\t%f\n", A.DT);
    fprintf(fchk, "PML REFLECTION COEFFICIENT:\t%f\n", A.ARBC);
    fprintf(fchk, "SKIP OF SEISMOGRAMS IN TIME (LOOP COUNTER):\t%d\n", A.NTISKP);
    fprintf(fchk, "ABC CONDITION, PML=1 OR CERJAN=0:\t%d\n", A.NPC);
    fprintf(fchk, "FD SCHEME, ELASTIC=0,VISCO=1,ELASTO-PLASTIC=2,VISCO-ELASTO-PLASTIC=3:\t%d\n",
            A.NVE);
    fprintf(fchk, "Q, FAC,Q0,EX,FP:\t%f, %f, %f, %f\n", A.FAC, A.Q0, A.EX, A.FP);
    fclose(fchk);
  }

  // ---- plasticity set-up per block (inidrpr_hoekbrown_light, mesh.c:1178-1401) --
  if (A.NVE == 3) {
    float strike[3] = {0, 0, 0}, dip[3] = {0, 90, 0}, fmajor = 0, fminor = 0, sigma_ci0 = 0,
          GSI = 0, mi = 0, gsi100 = 1;
    int sigma_ci_type = 0, fltpos = 0;
    FILE* fid = fopen("nonlinear.dat", "r");
    if (!fid) {
      perror("could not open nonlinear.dat");
      return 1;
    }
    char line[512];
    if (fgets(line, sizeof line, fid)) sscanf(line, "%f %f", strike, strike + 2);
    if (fgets(line, sizeof line, fid)) sscanf(line, "%f %f", &fmajor, &fminor);
    if (fgets(line, sizeof line, fid)) sscanf(line, "%d %f", &sigma_ci_type, &sigma_ci0);
    if (fgets(line, sizeof line, fid)) sscanf(line, "%f", &GSI);
    if (fgets(line, sizeof line, fid)) sscanf(line, "%f", &mi);
    if (fgets(line, sizeof line, fid)) sscanf(line, "%f", &gsi100);
    if (fgets(line, sizeof line, fid)) sscanf(line, "%d", &fltpos);
    fclose(fid);
    for (int p = 0; p < G; ++p) {
      std::vector<float> d1(ncell[p]), mu(ncell[p]), lam(ncell[p]), sigma2(ncell[p], 0.f),
          cohes(ncell[p], 0.f), phi(ncell[p], 0.f);
      AWP(awp_field_download(ctx[p], AWP_D1, d1.data()));
      AWP(awp_field_download(ctx[p], AWP_MU, mu.data()));
      AWP(awp_field_download(ctx[p], AWP_LAM, lam.data()));
      const long S = dims[p][1] * dims[p][2], Y = dims[p][2];
      auto at = [&](int i, int j, int k) { return (size_t)(i * S + j * Y + k); };
      const int nx = nxt[p], ny = nyt[p], nz = nzt[p];
      const int sInd = nz + ALIGN - 1;
      const float dh = DHp[p];
      float sigma_ci = sigma_ci0;
      for (int j = 2; j < ny + 2 + 2 * NGSL; j++)
        for (int i = 2; i < nx + 2 + 2 * NGSL; i++) {
          sigma2[at(i, j, sInd)] = -dh / 2. * d1[at(i, j, sInd)] * 9.81;
          sigma2[at(i, j, sInd + 1)] = sigma2[at(i, j, sInd)];
          for (int k = sInd - 1; k >= ALIGN - 2; k--)
            sigma2[at(i, j, k)] = sigma2[at(i, j, k + 1)] - dh * d1[at(i, j, k)] * 9.81;
        }
      for (int k = ALIGN; k <= sInd + 1; k++)
        for (int j = 2; j < ny + 2 + 2 * NGSL; j++)
          for (int i = 2; i < nx + 2 + 2 * NGSL; i++) {
            const float depth = 0.5 * dh + dh * (sInd - k);
            float GSI_wallrock = GSI + (100. - GSI) * (depth - 0.5 * dh) / gsi100, GSI_core,
                  GSI_d;
            if (GSI_wallrock > 100) GSI_wallrock = 100;
            if (depth < 4000.) GSI_core = GSI;
            else if (depth >= 4000. && depth <= 6000.)
              GSI_core = GSI + (depth - 4000.) / 2000. * (GSI_wallrock - GSI);
            else GSI_core = GSI_wallrock;
            const int ypos = j - 2 - NGSL;
            const float fltdist = fabsf((float)ypos + 0.5 - (float)fltpos) * dh;
            if (fltdist < 225.) GSI_d = GSI_core;
            else if (fltdist >= 225. && fltdist <= 750.)
              GSI_d = GSI_core + (GSI_wallrock - GSI_core) * (fltdist - 225.) / (750. - 225.);
            else GSI_d = GSI_wallrock;
            const size_t q = at(i, j, k);
            if (sigma_ci_type == 3) {
              const float tvp = sqrt((1. / lam[q] + 2. / mu[q]) / d1[q]);
              const float itime = 1. / tvp / 3.28 * 1.e6;
              sigma_ci = 1.4138e7 * powf(itime, -3.) * 1.e6;
            } else if (sigma_ci_type == 12) {
              const float tvp = sqrt((1. / lam[q] + 2. / mu[q]) / d1[q]) / 1.e3;
              sigma_ci = 0.77 * pow(tvp, 2.93) * 1.e6;
            }
            hoek_brown(-sigma2[q], sigma_ci, GSI_d, mi, 0, 1, &phi[q], &cohes[q]);
            const float tvs = sqrtf(1. / (mu[q] * d1[q]));
            if (tvs > 2000.) cohes[q] = 1.e12;
            else if (tvs < 750.) {
              cohes[q] = 0.f;
              phi[q] = 35.f;
            }
          }
      // no yielding around source nodes (pmcl3d.c:963-988)
      for (int s = 0; s < nsrc[p]; ++s) {
        const int idx = spos[p][3 * s] + 1 + NGSL, idy = spos[p][3 * s + 1] + 1 + NGSL;
        const int idz = (nz + 1 - spos[p][3 * s + 2]) + ALIGN - 1;
        for (int xi = idx - 1; xi < idx + 2; xi++)
          for (int yi = idy - 2; yi < idy + 2; yi++)
            for (int zi = idz - 1; zi < idz + 2; zi++) {
              const bool dox = xi >= 0 && xi < nx + 2 * NGSL + 1;
              const bool doy = yi >= 0 && yi < ny + 2 * NGSL + 1;
              const bool doz = zi >= 0 && yi < nz + 2 * NGSL + 1;
              if (dox && doy && doz) cohes[at(xi, yi, zi)] = 1.e18;
            }
      }
      AWP(awp_upload_plasticity(ctx[p], sigma2.data(), cohes.data(), phi.data(), fmajor, fminor,
                                strike, dip));
    }
  }

  // ---- curvilinear topography of grid 0 (pmcl3d.c:1522-1548) --------------------
  if (A.USETOPO) AWP(awp_topography_init(ctx[0], A.INTOPO.c_str()));

  // ---- SOURCEFILE / RECVFILE / SGTFILE point sets (pmcl3d.c:1563-1578, 1603-1607) -
  if (A.USESOURCEFILE) AWP(awp_sourcefile_init(ctx[0], A.SOURCEFILE.c_str()));
  if (A.USERECVFILE) AWP(awp_receivers_init(ctx[0], A.RECVFILE.c_str(), nt));
  // FORCEFILE boundary forces (pmcl3d.c:1569-1571, 1608, 1989-1994): added in
  // the curvilinear branch of the time loop only, so without topography the
  // reference reads them and never applies them
  if (A.USEFORCEFILE) {
    if (A.USETOPO) AWP(awp_forcefile_init(ctx[0], A.FORCEFILE.c_str()));
    else printf("FORCEFILE %s: forces act with topography only; not applied\n",
                A.FORCEFILE.c_str());
  }
  // SGTFILE stress receivers and material output (pmcl3d.c:1572-1578, 1605)
  if (A.USESGTFILE) AWP(awp_sgt_init(ctx[0], A.SGTFILE.c_str(), nt));

  // ---- output buffers ------------------------------------------------------------
  size_t rec[MAXGRIDS];
  std::vector<float> Bufx[MAXGRIDS], Bufy[MAXGRIDS], Bufz[MAXGRIDS], Bufeta[MAXGRIDS];
  float *d_bx[MAXGRIDS] = {}, *d_by[MAXGRIDS] = {}, *d_bz[MAXGRIDS] = {}, *d_be[MAXGRIDS] = {};
  for (int p = 0; p < G; ++p) {
    rec[p] = (size_t)rnx[p] * rny[p] * rnz[p];
    Bufx[p].resize(rec[p] * A.WRITE_STEP);
    Bufy[p].resize(rec[p] * A.WRITE_STEP);
    Bufz[p].resize(rec[p] * A.WRITE_STEP);
    Bufeta[p].resize(A.NVE == 3 ? rec[p] * A.WRITE_STEP : 0);
    if (rec[p]) {
      // the gather writes straight into host-visible pinned memory
      AWP(awp_alloc_host_pinned((void**)&d_bx[p], rec[p] * sizeof(float)));
      AWP(awp_alloc_host_pinned((void**)&d_by[p], rec[p] * sizeof(float)));
      AWP(awp_alloc_host_pinned((void**)&d_bz[p], rec[p] * sizeof(float)));
      if (A.NVE == 3) AWP(awp_alloc_host_pinned((void**)&d_be[p], rec[p] * sizeof(float)));
    }
  }
  mkdir(A.OUT.c_str(), 0755);
  fchk = fopen(A.CHKFILE.c_str(), "a+");
  auto step_all = [&](int n) {
    if (mesh) AWP(awp_mesh_step(mesh, n));
    else AWP(awp_step(ctx[0], n));
  };
  auto sync_all = [&]() {
    if (mesh) AWP(awp_mesh_synchronize(mesh));
    else AWP(awp_synchronize(ctx[0]));
  };

  time_init = now() - time_init;
  printf("Initialization completed in %f s.\n", time_init);
  printf("Time step \t Time \t\t Elapsed time \t sec per time step \t Time steps per sec \t "
         "Percentage completed\n");
  printf("---------------------------------------------------------------------------------"
         "------------------------------------\n");
  double time_un = 0;
  long cur_step = 0;
  if ((A.NPC == 0 || A.NPC == 2) && (A.NVE == 1 || A.NVE == 3)) {
    time_un -= now();
    for (cur_step = 1; cur_step <= nt; cur_step++) {
      step_all(1);
      if (cur_step % 10 == 0) {
        sync_all();
        const double elapsed = now() + time_un;
        const double step_s = elapsed / cur_step;
        printf("%ld  \t\t %4.3f s \t %4.3f s \t %3.5f s/step \t %5.3f step/s \t %2.2f %%  \n",
               cur_step, cur_step * A.DT, elapsed, step_s, 1.0 / step_s,
               100 * (double)cur_step / (double)(nt - 1));
        fflush(stdout);
      }
      if (cur_step % A.NTISKP == 0) {
        for (int p = 0; p < G; ++p) {
          if (!rec[p]) continue;
          AWP(awp_gather_output(ctx[p], rnbgx[p], rnedx[p], A.NSKPX[p], rnbgy[p], rnedy[p],
                                A.NSKPY[p], rnbgz[p], rnedz[p], A.NSKPZ[p], d_bx[p], d_by[p],
                                d_bz[p], d_be[p]));
          sync_all();
          const long idtmp = ((cur_step / A.NTISKP + A.WRITE_STEP - 1) % A.WRITE_STEP) * rec[p];
          memcpy(Bufx[p].data() + idtmp, d_bx[p], rec[p] * 4);
          memcpy(Bufy[p].data() + idtmp, d_by[p], rec[p] * 4);
          memcpy(Bufz[p].data() + idtmp, d_bz[p], rec[p] * 4);
          if (A.NVE == 3) memcpy(Bufeta[p].data() + idtmp, d_be[p], rec[p] * 4);
        }
        for (int p = 0; p < G; ++p) {
          if ((cur_step / A.NTISKP) % A.WRITE_STEP != 0 || !rec[p]) continue;
          // file view of pmcl3d.c:489-521 at one rank: WRITE_STEP x rec_NZ x
          // rec_NY x rec_NX floats, this rank's rec_nzt x rec_nyt x rec_nxt
          // points at the origin (rows beyond them stay empty)
          const char* base[4] = {"SX", "SY", "SZ", "Eta"};
          std::vector<float>* bufs[4] = {&Bufx[p], &Bufy[p], &Bufz[p], &Bufeta[p]};
          const size_t fsz = (size_t)A.WRITE_STEP * recNZ[p] * recNY[p] * recNX[p];
          std::vector<float> file(fsz);
          for (int c = 0; c < (A.NVE == 3 ? 4 : 3); ++c) {
            std::fill(file.begin(), file.end(), 0.f);
            const float* b = bufs[c]->data();
            for (int t = 0; t < A.WRITE_STEP; ++t)
              for (int z = 0; z < rnz[p]; ++z)
                for (int y = 0; y < rny[p]; ++y)
                  memcpy(&file[(((size_t)t * recNZ[p] + z) * recNY[p] + y) * recNX[p]],
                         b + (((size_t)t * rnz[p] + z) * rny[p] + y) * rnx[p],
                         rnx[p] * sizeof(float));
            char fn[600];
            snprintf(fn, sizeof fn, "%s/%s_%1d_%07ld", A.OUT.c_str(), base[c], p, cur_step);
            FILE* fo = fopen(fn, "wb");
            if (!fo) die("open output", AWP_ERR_IO);
            fwrite(file.data(), sizeof(float), fsz, fo);
            fclose(fo);
          }
        }
        // statistics line (pmcl3d.c:2426-2437): the reference prints its host
        // copies of u1/v1/w1, which are never refreshed from the device, so the
        // values are the initial zeros
        if (fchk) {
          fprintf(fchk, "%ld :\t%e\t%e\t%e\n", cur_step, 0.0, 0.0, 0.0);
          fflush(fchk);
        }
      }
    }
    sync_all();
    time_un += now();
  }
  if (A.IFAULT == 5) {
    float tmom = 0.0f;
    for (int p = 0; p < G; ++p) {
      if (!nsrc[p]) continue;
      std::vector<float> mom(nsrc[p]);
      AWP(awp_download_moment(ctx[p], mom.data()));
      for (float m : mom) tmom += m;
    }
    if (tmom != 0.0f) {
      printf("rank %d: moment=%e\n", 0, tmom);
      const float mag = 2. / 3. * (log10f(tmom) - 9.1);
      printf("Total M0=%e, Mw=%4.1f\n", tmom, mag);
    }
  }
  if (fchk) {
    fprintf(fchk, "END\n");
    fclose(fchk);
  }
  long long cells = 0;
  for (int p = 0; p < G; ++p) cells += (long long)nxt[p] * nyt[p] * nzt[p];
  if (nt > 0 && cur_step > 1)
    printf("%ld steps in %.3f s: %.6f s per time step, %.3f Gcell-updates/s\n", cur_step - 1,
           time_un, time_un / (cur_step - 1), (double)cells * (cur_step - 1) / time_un / 1e9);
  for (int p = 0; p < G; ++p) {
    if (d_bx[p]) awp_free_host_pinned(d_bx[p]);
    if (d_by[p]) awp_free_host_pinned(d_by[p]);
    if (d_bz[p]) awp_free_host_pinned(d_bz[p]);
    if (d_be[p]) awp_free_host_pinned(d_be[p]);
  }
  if (mesh) awp_mesh_destroy(mesh);
  else awp_ctx_destroy(ctx[0]);
  return 0;
}
