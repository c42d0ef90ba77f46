// diag.cu -- diagnostics of the reference driver's output steps
// (Source1.f90:218-234): the field dump output_results (:898-924), the
// per-particle log output_result2 (:1420-1441), the neck file of output3
// (:1673-1717) and the energy budget output4 (:1719-1797).
//
// The sums are reduced on the device in a fixed order (deterministic); the
// files are Tecplot ASCII with the reference's variables and number formats.
// Departures, each a fix of the reference:
//   - output4 indexes walls_all(z,y,z), rho(z,y,z) and uz(z,y,z) (:1736,
//     :1739); the sums here use (z,y,x);
//   - the reference re-opens P_pp.dat, hmin.dat and Energy.dat on every call
//     without position='append', so each keeps only its last record; the
//     writers here append one record per call (the header at t = 0).
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>
#include "state.cuh"

using namespace symb200;

namespace {

constexpr int kT = 256;

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
#pragma unroll
  for (int s = NT / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// output4 field sums (:1729-1750): pressure energy (rho - rho0)/3 and kinetic
// energy rho |u|^2 / 2 over red fluid nodes, and the number of fluid nodes
// with a fluid neighbour of the other colour (the interface area).  REFERENCE
// geometry: interior nodes 2..n-1 (1-based) with in-range neighbours; CONFIG:
// every node, periodic neighbours.
__global__ void k_energy(DevParams P, const double* __restrict__ rho, const double* __restrict__ ux,
                         const double* __restrict__ uy, const double* __restrict__ uz,
                         const double* __restrict__ rhoN, const int32_t* __restrict__ walls_all, double* part) {
  __shared__ double sh[kT];
  const long long L = blockIdx.x * (long long)kT + threadIdx.x;
  double v[3] = {0.0, 0.0, 0.0};
  if (L < P.N) {
    const int z = (int)(L % P.nz), y = (int)((L / P.nz) % P.ny), x = (int)(L / ((long long)P.nz * P.ny));
    const bool in = !P.ref || (x >= 1 && x <= P.nx - 2 && y >= 1 && y <= P.ny - 2 && z >= 1 && z <= P.nz - 2);
    if (in && walls_all[L] <= 0) {
      if (rhoN[L] > 0.0) {
        v[0] = (rho[L] - P.rho0) / 3.0;
        v[1] = 0.5 * rho[L] * (ux[L] * ux[L] + uy[L] * uy[L] + uz[L] * uz[L]);
      }
      for (int i = 1; i < 19; i++) {
        const int xn = P.ref ? x + CX(i) : wrapi(x + CX(i), P.nx);
        const int yn = P.ref ? y + CY(i) : wrapi(y + CY(i), P.ny);
        const int zn = P.ref ? z + CZ(i) : wrapi(z + CZ(i), P.nz);
        const long long Ln = lin(P, xn, yn, zn);
        if (rhoN[L] * rhoN[Ln] < 0.0 && walls_all[Ln] <= 0) {
          v[2] = 1.0;
          break;
        }
      }
    }
  }
  for (int k = 0; k < 3; k++) {
    const double s = block_sum<kT>(v[k], sh);
    if (threadIdx.x == 0) part[blockIdx.x * 3LL + k] = s;
  }
}
__global__ void k_energy_final(const double* part, long long nblk, double* out) {
  __shared__ double sh[kT];
  for (int k = 0; k < 3; k++) {
    double s = 0.0;
    for (long long b = threadIdx.x; b < nblk; b += kT) s += part[b * 3 + k];
    s = block_sum<kT>(s, sh);
    if (threadIdx.x == 0) out[k] = s;
  }
}

// the macroscopic fields of the current populations (calmacros) in the
// canonical arrays, without changing the stepping state
int macros(sym_handle* h) { return current_macros(h); }

// output4's halving of a particle that starts on a mirror plane (:1765-1779)
double mirror_factor(const sym_handle* h, const sym_particles& s, int pp) {
  if (!h->dp.ref) return 1.0;
  const int par = h->dp.par;
  auto c0 = [&](int k) { return s.center0[k * par + pp - 1]; };
  double f = 1.0;
  if (std::fabs(c0(1) - ((double)h->dp.ny - 0.5)) < 0.1 || std::fabs(c0(1) - 1.5) < 0.1) f *= 0.5;
  if (std::fabs(c0(0) - ((double)h->dp.nx - 0.5)) < 0.1) f *= 0.5;
  if (std::fabs(c0(2) - ((double)h->dp.nz - 0.5)) < 0.1) f *= 0.5;
  return f;
}

FILE* open_log(sym_handle* h, const std::string& path, int t) {
  FILE* f = fopen(path.c_str(), t == 0 ? "w" : "a");
  if (!f) set_error(h, SYM_ERR_PARAM, "cannot open %s", path.c_str());
  return f;
}

}  // namespace

extern "C" {

int sym_energy(sym_handle* h, double out[6]) {
  if (!h || !out) return SYM_ERR_PARAM;
  if (int e = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice")) return e;
  if (int e = macros(h)) return e;
  const DevParams& P = h->dp;
  const long long nblk = (P.N + kT - 1) / kT;
  if ((size_t)(nblk * 3 + 8) > h->red_len) return set_error(h, SYM_ERR_STATE, "reduction scratch too small");
  k_energy<<<(unsigned)nblk, kT, 0, h->st>>>(P, h->rho, h->ux, h->uy, h->uz, h->rhoN, h->walls_all, h->red);
  k_energy_final<<<1, kT, 0, h->st>>>(h->red, nblk, h->red + nblk * 3);
  double f[3];
  cudaMemcpyAsync(f, h->red + nblk * 3, sizeof f, cudaMemcpyDeviceToHost, h->st);
  sym_particles s;
  cudaMemcpyAsync(&s, h->dpart, sizeof s, cudaMemcpyDeviceToHost, h->st);
  if (int e = check_cuda(h, cudaStreamSynchronize(h->st), "energy")) return e;
  // particle terms (:1757-1781)
  double emp = 0.0, wcap = 0.0, shb = 0.0;
  const int par = P.par;
  for (int pp = 1; pp <= par; pp++) {
    auto A = [&](const double* a, int k) { return a[k * par + pp - 1]; };
    double e = 0.5 * P.mass * (A(s.up, 0) * A(s.up, 0) + A(s.up, 1) * A(s.up, 1) + A(s.up, 2) * A(s.up, 2)) +
               0.5 * P.inertia * (A(s.rp, 0) * A(s.rp, 0) + A(s.rp, 1) * A(s.rp, 1) + A(s.rp, 2) * A(s.rp, 2));
    double w = A(s.tension, 0) * A(s.up, 0) + A(s.tension, 1) * A(s.up, 1) + A(s.tension, 2) * A(s.up, 2) +
               A(s.tension_t, 0) * A(s.rp, 0) + A(s.tension_t, 1) * A(s.rp, 1) + A(s.tension_t, 2) * A(s.rp, 2);
    double a = s.shb[pp - 1];
    const double m = mirror_factor(h, s, pp);
    emp += e * m;
    wcap += w * m;
    shb += a * m;
  }
  out[0] = f[0]; out[1] = f[1]; out[2] = f[2];
  out[3] = emp; out[4] = wcap; out[5] = shb;
  return SYM_OK;
}

int sym_output_results(sym_handle* h, const char* path) {
  if (!h || !path) return SYM_ERR_PARAM;
  if (int e = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice")) return e;
  if (int e = macros(h)) return e;
  const size_t N = h->N;
  std::vector<double> rho(N), ux(N), uy(N), uz(N), rn(N);
  std::vector<int32_t> wa(N);
  cudaMemcpyAsync(rho.data(), h->rho, 8 * N, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(ux.data(), h->ux, 8 * N, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(uy.data(), h->uy, 8 * N, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(uz.data(), h->uz, 8 * N, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(rn.data(), h->rhoN, 8 * N, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(wa.data(), h->walls_all, 4 * N, cudaMemcpyDeviceToHost, h->st);
  if (int e = check_cuda(h, cudaStreamSynchronize(h->st), "output_results")) return e;
  FILE* f = fopen(path, "w");
  if (!f) return set_error(h, SYM_ERR_PARAM, "cannot open %s", path);
  const int nx = h->dp.nx, ny = h->dp.ny, nz = h->dp.nz;
  fprintf(f, " TITLE=\"Contact_Angles\"\n VARIABLES=X,Y,Z,WALL,RHO_N,U,V,W,RHO\n");
  fprintf(f, " ZONE F=POINT I=%12d J=%12d K=%12d\n", nx, ny, nz);
  std::string buf;
  buf.reserve(1 << 20);
  char line[160];
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        const size_t L = (size_t)z + (size_t)nz * ((size_t)y + (size_t)ny * (size_t)x);
        const int n = snprintf(line, sizeof line, " %6d %6d %6d %6d %12.8f %12.8f %12.8f %12.8f %12.8f\n", x + 1,
                               y + 1, z + 1, wa[L], rn[L], ux[L], uy[L], uz[L], rho[L]);
        buf.append(line, (size_t)n);
        if (buf.size() > (1u << 20)) {
          fwrite(buf.data(), 1, buf.size(), f);
          buf.clear();
        }
      }
  fwrite(buf.data(), 1, buf.size(), f);
  const bool ok = fclose(f) == 0;
  return ok ? SYM_OK : set_error(h, SYM_ERR_PARAM, "write to %s failed", path);
}

int sym_output_result2(sym_handle* h, const char* prefix, int t, double tr) {
  if (!h || !prefix) return SYM_ERR_PARAM;
  if (int e = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice")) return e;
  sym_particles s;
  if (int e = check_cuda(h, cudaMemcpy(&s, h->dpart, sizeof s, cudaMemcpyDeviceToHost), "output_result2")) return e;
  const int par = h->dp.par;
  for (int pp = 1; pp <= par; pp++) {
    FILE* f = open_log(h, std::string(prefix) + "P_" + std::to_string(pp) + ".dat", t);
    if (!f) return SYM_ERR_PARAM;
    if (t == 0)
      fprintf(f, " VARIABLES=t,t*,cx,cy,cz,upx,upy,upz,rpx,rpy,rpz,Fpx,Fpy,Fpz,Tpx,Tpy,Tpz,Fcx,Fcy,Fcz,Tcx,Tcy,Tcz,"
                 "Frex,Frey,Frez\n");
    auto A = [&](const double* a, int k) { return a[k * par + pp - 1]; };
    fprintf(f, " %6d %12.6f", t, (double)t / tr);
    const double* arr[8] = {s.center, s.up, s.rp, s.fp, s.tp, s.tension, s.tension_t, s.fre};
    for (const double* a : arr)
      for (int k = 0; k < 3; k++) fprintf(f, " %12.6f", A(a, k));
    fprintf(f, "\n");
    if (fclose(f) != 0) return set_error(h, SYM_ERR_PARAM, "write of P_%d.dat failed", pp);
  }
  return SYM_OK;
}

int sym_output3_write(sym_handle* h, const char* path, int t, double tr, double rad_c, double lamda_d) {
  if (!h || !path) return SYM_ERR_PARAM;
  double hmin = 0.0;
  int32_t y0 = 0;
  if (int e = sym_output3(h, &hmin, &y0)) return e;
  FILE* f = open_log(h, path, t);
  if (!f) return SYM_ERR_PARAM;
  if (t == 0) fprintf(f, " VARIABLES=t,t*,h,y0\n");
  fprintf(f, " %8d %12.6f %12.6f %12.6f\n", t, (double)t / tr, hmin / rad_c, (double)y0 / lamda_d);
  return fclose(f) == 0 ? SYM_OK : set_error(h, SYM_ERR_PARAM, "write to %s failed", path);
}

int sym_output4(sym_handle* h, const char* path, int t, double tr, double rad_c, double* wcap_acc) {
  if (!h || !path || !wcap_acc) return SYM_ERR_PARAM;
  double e[6];
  if (int rc = sym_energy(h, e)) return rc;
  // normalisation of :1751-1787: energies by pi Rc^2 sigma, the 1/8 domain of
  // the reference geometry counted 8 times
  const double oct = h->dp.ref ? 8.0 : 1.0;
  const double er = M_PI * rad_c * rad_c * h->dp.sigma;
  const double epv = e[0] / er * oct, emov = e[1] / er * oct, esur = e[2] / 2.0 * h->dp.sigma / er * oct;
  const double emp = e[3] / er * oct;
  *wcap_acc = *wcap_acc + e[4] / er * oct;
  const double shb = e[5] / (M_PI * rad_c * rad_c) * oct;
  FILE* f = open_log(h, path, t);
  if (!f) return SYM_ERR_PARAM;
  if (t == 0) fprintf(f, " VARIABLES=t,t*,Esur,Shb,Efree,Emov,Wcap,Emov_p,Esum\n");
  fprintf(f, " %8d %12.6f %12.6f %12.6f %12.6f %12.6f %12.6f %12.6f %12.6f\n", t, (double)t / tr, esur, shb,
          esur - epv, emov, *wcap_acc, emp, esur - epv + emov + emp);
  return fclose(f) == 0 ? SYM_OK : set_error(h, SYM_ERR_PARAM, "write to %s failed", path);
}

}  // extern "C"
