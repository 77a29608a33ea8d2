// Test infrastructure: command-line front end of the reference driver (ref_driver.cpp).
// The reference library is run in its own process and fed through raw little-endian
// files: loaded into a Python process with ctypes, its host-side runtime intermittently
// blocked on a futex before the first operator launch, while the same calls from a plain
// C/C++ process never did.  Usage:  zsref_cli <request file> <reply file>
//
// Request: int32 command, then
//   1 run:       zsref_params, int32 n, int32 nsteps, int32 cap_blocks,
//                f32 m[n], x[3n], v[3n], C[9n], F[9n], logJp[n]
//     reply:     int32 status, int32 nblocks, f64 seconds, x, v, C, F, logJp,
//                int32 keys[3*nblocks], f32 grid[nblocks*4*512]   (keys/grid if status==0)
//   2 activate:  int32 n, f32 dx, int32 table_expected, int32 cap, f32 x[3n]
//     reply:     int32 status, nblocks, nparblocks, table_size, keys[3*nb], slots[nb]
//   3 stress:    int32 count, int32 model, f32 volume, E, nu, friction_deg, cohesion, beta,
//                int32 volume_correction, f32 F[9*count], logJp[count]
//     reply:     f32 PF[9*count], F[9*count], logJp[count]
//   4 svd:       int32 count, f32 A[9*count]
//     reply:     f32 U[9*count], S[3*count], V[9*count]
//   5 bht:       int32 nkeys, int32 expected, int32 cap_slots, int32 keys[3*nkeys]
//     reply:     int32 status, table_size, u32 hash[6], int32 cnt,
//                then (status == 0) int32 keys[3*table_size], indices[table_size], status[table_size]
//   6 g2p2g:     zsref_params, int32 n, int32 nb, f32 x[3n], F[9n], logJp[n],
//                int32 keys[3*nb], f32 v[1536*nb]
//     reply:     int32 status, f64 seconds, then (status == 0) f32 f[1536*nb]
//   8 run with colliders: as 1, then int32 ncolliders and ncolliders zsmpm_collider records
//     reply:     as 1
//   9 run with colliders and sparse level sets: as 8, then int32 nlevelsets and per level set
//                int32 nblocks, type, f32 background, sinv[9], rinv[9], t[3],
//                int32 keys[3*nblocks], f32 sdf[512*nblocks]
//     reply:     as 1
//  10 run with the cell-centric transfers (P2C2G / G2C2P): as 1
//     reply:     as 1 (logJp unchanged)
//   7 implicit:  zsref_params, int32 op, n, nb, max_iters, f32 tol, rel_tol,
//                f32 m[n], x[3n], v[3n], C[9n], F[9n], logJp[n], int32 keys[3*nb],
//                f32 a[1536*nb], b[1536*nb]
//     reply:     int32 status, int32 iters, f64 seconds, then (status == 0)
//                f32 out[1536*nb], mass[512*nb]
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "zeroed_new.hpp"  // the reference registry's mutex starts unlocked

extern "C" {
struct zsref_params {
  int model, policy, threads, order, wall_type, wall_cells, table_expected, volume_correction;
  float dx, dt, gx, gy, gz;
  float E, nu, volume;
  float friction_deg, cohesion, beta;
};
int zsref_run(const zsref_params *p, int n, float *m, float *x, float *v, float *C, float *F,
              float *logJp, int nsteps, int cap_blocks, int *out_nblocks, int *out_keys,
              float *out_grid, double *out_seconds);
int zsref_run_colliders(const zsref_params *p, int n, float *m, float *x, float *v, float *C, float *F,
                        float *logJp, int nsteps, int cap_blocks, int *out_nblocks, int *out_keys,
                        float *out_grid, double *out_seconds, int ncolliders, const void *colliders,
                        int nlevelsets, const void *levelsets);
int zsref_run_cell(const zsref_params *p, int n, float *m, float *x, float *v, float *C, float *F,
                   int nsteps, int cap_blocks, int *out_nblocks, int *out_keys, float *out_grid,
                   double *out_seconds);
// the driver's ref_levelset record
struct ref_levelset_rec {
  int nblocks, type;
  float background, sinv[9], rinv[9], t[3];
  const int *keys;
  const float *sdf;
};
void zsref_stress(int model, float volume, float E, float nu, float friction_deg,
                  float cohesion, float beta, int volume_correction, float *F, float *logJp,
                  float *PF);
void zsref_svd(const float *A, float *U, float *S, float *V);
int zsref_activate(int n, const float *x, float dx, int table_expected, int cap,
                   int *out_nblocks, int *out_nparblocks, int *out_keys, int *out_slots,
                   int *out_table_size);
int zsref_bht(int nkeys, const int *keys, int expected, int cap_slots, int *out_table_size,
              unsigned *out_hash, int *out_keys, int *out_indices, int *out_status, int *out_cnt);
int zsref_g2p2g(const zsref_params *p, int n, const float *x, const float *F, const float *logJp,
                int nb_expected, const int *keys, const float *vin, float *fout,
                double *out_seconds);
int zsref_implicit(const zsref_params *p, int op, int n, const float *m, const float *x, const float *v,
                   const float *C, const float *F, const float *logJp, int nb_expected, const int *keys,
                   const float *a, const float *b, int max_iters, float tol, float rel_tol, float *out,
                   float *out_mass, int *iters, double *out_seconds);
}

namespace {
  FILE *in_f, *out_f;
  template <typename T> T rd() {
    T v{};
    if (std::fread(&v, sizeof(T), 1, in_f) != 1) {
      std::fprintf(stderr, "zsref_cli: short request\n");
      std::exit(3);
    }
    return v;
  }
  template <typename T> void rdv(std::vector<T> &v, size_t n) {
    v.resize(n);
    if (n && std::fread(v.data(), sizeof(T), n, in_f) != n) {
      std::fprintf(stderr, "zsref_cli: short request array\n");
      std::exit(3);
    }
  }
  template <typename T> void wr(const T &v) { std::fwrite(&v, sizeof(T), 1, out_f); }
  template <typename T> void wrv(const T *p, size_t n) {
    if (n) std::fwrite(p, sizeof(T), n, out_f);
  }
}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: zsref_cli <request> <reply>\n");
    return 2;
  }
  in_f = std::fopen(argv[1], "rb");
  out_f = std::fopen(argv[2], "wb");
  if (!in_f || !out_f) return 2;
  const int cmd = rd<int32_t>();
  if (cmd == 1 || cmd == 8 || cmd == 9 || cmd == 10) {
    auto p = rd<zsref_params>();
    const int n = rd<int32_t>(), nsteps = rd<int32_t>(), cap = rd<int32_t>();
    std::vector<float> m, x, v, C, F, lj;
    rdv(m, n);
    rdv(x, 3 * (size_t)n);
    rdv(v, 3 * (size_t)n);
    rdv(C, 9 * (size_t)n);
    rdv(F, 9 * (size_t)n);
    rdv(lj, n);
    int ncol = 0;
    std::vector<unsigned char> cols;
    if (cmd == 8 || cmd == 9) {
      ncol = rd<int32_t>();
      rdv(cols, (size_t)ncol * 120);  // 4 int32 + 26 float32 per collider
    }
    int nls = 0;
    std::vector<ref_levelset_rec> lss;
    std::vector<std::vector<int>> ls_keys;
    std::vector<std::vector<float>> ls_sdf;
    if (cmd == 9) {
      nls = rd<int32_t>();
      lss.resize(nls);
      ls_keys.resize(nls);
      ls_sdf.resize(nls);
      for (int k = 0; k < nls; ++k) {
        ref_levelset_rec &L = lss[k];
        L.nblocks = rd<int32_t>();
        L.type = rd<int32_t>();
        L.background = rd<float>();
        for (float &f : L.sinv) f = rd<float>();
        for (float &f : L.rinv) f = rd<float>();
        for (float &f : L.t) f = rd<float>();
        rdv(ls_keys[k], 3 * (size_t)L.nblocks);
        rdv(ls_sdf[k], 512 * (size_t)L.nblocks);
        L.keys = ls_keys[k].data();
        L.sdf = ls_sdf[k].data();
      }
    }
    std::vector<int> keys(3 * (size_t)cap);
    std::vector<float> grid((size_t)cap * 4 * 512);
    int nb = 0;
    double secs = 0;
    int st = cmd == 10 ? zsref_run_cell(&p, n, m.data(), x.data(), v.data(), C.data(), F.data(), nsteps, cap,
                                        &nb, cap ? keys.data() : nullptr, cap ? grid.data() : nullptr, &secs)
                       : zsref_run_colliders(&p, n, m.data(), x.data(), v.data(), C.data(), F.data(), lj.data(),
                                             nsteps, cap, &nb, cap ? keys.data() : nullptr,
                                             cap ? grid.data() : nullptr, &secs, ncol, cols.data(), nls, lss.data());
    wr<int32_t>(st);
    wr<int32_t>(nb);
    wr<double>(secs);
    wrv(x.data(), x.size());
    wrv(v.data(), v.size());
    wrv(C.data(), C.size());
    wrv(F.data(), F.size());
    wrv(lj.data(), lj.size());
    if (st == 0 && cap) {
      wrv(keys.data(), 3 * (size_t)nb);
      wrv(grid.data(), (size_t)nb * 4 * 512);
    }
  } else if (cmd == 2) {
    const int n = rd<int32_t>();
    const float dx = rd<float>();
    const int expected = rd<int32_t>(), cap = rd<int32_t>();
    std::vector<float> x;
    rdv(x, 3 * (size_t)n);
    std::vector<int> keys(3 * (size_t)cap), slots(cap);
    int nb = 0, npb = 0, ts = 0;
    int st = zsref_activate(n, x.data(), dx, expected, cap, &nb, &npb, keys.data(),
                            slots.data(), &ts);
    wr<int32_t>(st);
    wr<int32_t>(nb);
    wr<int32_t>(npb);
    wr<int32_t>(ts);
    if (st == 0) {
      wrv(keys.data(), 3 * (size_t)nb);
      wrv(slots.data(), (size_t)nb);
    }
  } else if (cmd == 3) {
    const int count = rd<int32_t>(), model = rd<int32_t>();
    const float vol = rd<float>(), E = rd<float>(), nu = rd<float>(), fa = rd<float>(),
                coh = rd<float>(), beta = rd<float>();
    const int vc = rd<int32_t>();
    std::vector<float> F, lj, PF(9 * (size_t)count);
    rdv(F, 9 * (size_t)count);
    rdv(lj, count);
    for (int i = 0; i != count; ++i)
      zsref_stress(model, vol, E, nu, fa, coh, beta, vc, &F[9 * (size_t)i], &lj[i],
                   &PF[9 * (size_t)i]);
    wrv(PF.data(), PF.size());
    wrv(F.data(), F.size());
    wrv(lj.data(), lj.size());
  } else if (cmd == 5) {
    const int nk = rd<int32_t>(), expected = rd<int32_t>(), cap = rd<int32_t>();
    std::vector<int> keys;
    rdv(keys, 3 * (size_t)nk);
    std::vector<int> tk(3 * (size_t)cap), ti(cap), tst(cap);
    unsigned hash[6] = {};
    int ts = 0, cnt = 0;
    int st = zsref_bht(nk, keys.data(), expected, cap, &ts, hash, tk.data(), ti.data(), tst.data(), &cnt);
    wr<int32_t>(st);
    wr<int32_t>(ts);
    wrv(hash, 6);
    wr<int32_t>(cnt);
    if (st == 0) {
      wrv(tk.data(), 3 * (size_t)ts);
      wrv(ti.data(), (size_t)ts);
      wrv(tst.data(), (size_t)ts);
    }
  } else if (cmd == 6) {
    auto p = rd<zsref_params>();
    const int n = rd<int32_t>(), nb = rd<int32_t>();
    std::vector<float> x, F, lj, v;
    std::vector<int> keys;
    rdv(x, 3 * (size_t)n);
    rdv(F, 9 * (size_t)n);
    rdv(lj, n);
    rdv(keys, 3 * (size_t)nb);
    rdv(v, 1536 * (size_t)nb);
    std::vector<float> f(1536 * (size_t)nb);
    double secs = 0;
    int st = zsref_g2p2g(&p, n, x.data(), F.data(), lj.data(), nb, keys.data(), v.data(), f.data(), &secs);
    wr<int32_t>(st);
    wr<double>(secs);
    if (st == 0) wrv(f.data(), f.size());
  } else if (cmd == 7) {
    auto p = rd<zsref_params>();
    const int op = rd<int32_t>(), n = rd<int32_t>(), nb = rd<int32_t>(), max_iters = rd<int32_t>();
    const float tol = rd<float>(), rel_tol = rd<float>();
    std::vector<float> m, x, v, C, F, lj, a, b;
    std::vector<int> keys;
    rdv(m, n);
    rdv(x, 3 * (size_t)n);
    rdv(v, 3 * (size_t)n);
    rdv(C, 9 * (size_t)n);
    rdv(F, 9 * (size_t)n);
    rdv(lj, n);
    rdv(keys, 3 * (size_t)nb);
    rdv(a, 1536 * (size_t)nb);
    rdv(b, 1536 * (size_t)nb);
    std::vector<float> out(1536 * (size_t)nb), mass(512 * (size_t)nb);
    int iters = 0;
    double secs = 0;
    int st = zsref_implicit(&p, op, n, m.data(), x.data(), v.data(), C.data(), F.data(), lj.data(), nb,
                            keys.data(), a.data(), b.data(), max_iters, tol, rel_tol, out.data(), mass.data(),
                            &iters, &secs);
    wr<int32_t>(st);
    wr<int32_t>(iters);
    wr<double>(secs);
    if (st == 0) {
      wrv(out.data(), out.size());
      wrv(mass.data(), mass.size());
    }
  } else if (cmd == 4) {
    const int count = rd<int32_t>();
    std::vector<float> A, U(9 * (size_t)count), S(3 * (size_t)count), V(9 * (size_t)count);
    rdv(A, 9 * (size_t)count);
    for (int i = 0; i != count; ++i)
      zsref_svd(&A[9 * (size_t)i], &U[9 * (size_t)i], &S[3 * (size_t)i], &V[9 * (size_t)i]);
    wrv(U.data(), U.size());
    wrv(S.data(), S.size());
    wrv(V.data(), V.size());
  } else {
    std::fprintf(stderr, "zsref_cli: unknown command %d\n", cmd);
    return 2;
  }
  std::fclose(out_f);
  return 0;
}
