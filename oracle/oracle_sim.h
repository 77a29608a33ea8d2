/* Test infrastructure (oracle): the substep restatement, written once and instantiated
 * for float (SFX=_f32) and double (SFX=_f64) by oracle.c.  Every expression keeps the
 * reference's operand order (the FP32 instance is pinned bit-exactly against the compiled
 * reference under a sequential schedule); see oracle.h for the file:line list.
 *
 * Required macros: R (float or double), SFX, R_LOG/R_EXP/R_SQRT/R_FLOOR/R_ABS (logf/expf/
 * sqrtf/floorf/fabsf or their double forms), OR_SVD (oracle_svd_f32 / oracle_svd_f64).
 */
#define OR_CAT2(a, b) a##b
#define OR_CAT(a, b) OR_CAT2(a, b)
#define OR_NAME(base) OR_CAT(base, SFX)

/* ConstitutiveModel.hpp:34-38.  The reference evaluates mu with a double literal 0.5,
 * so for T=float mu = float(0.5 * double(E) / double(1 + nu)); lambda stays in T. */
static void OR_NAME(lame)(R E, R nu, R *mu, R *lam) {
  *mu = (R)(0.5 * (double)E / (double)((R)1 + nu));
  *lam = E * nu / (((R)1 + nu) * ((R)1 - (R)2 * nu));
}

/* out[3c+r] = sum_k U[3k+r] d[k] V[3k+c], products as ((U d) V)  (MatrixUtils.h:26-45) */
static void OR_NAME(mat_diag_matT)(R *out, const R *U, const R *d, const R *V) {
  for (int c = 0; c != 3; ++c)
    for (int r = 0; r != 3; ++r)
      out[3 * c + r] = U[r] * d[0] * V[c] + U[3 + r] * d[1] * V[3 + c] +
                       U[6 + r] * d[2] * V[6 + c];
}

/* PF[3c+r] = (sum_k P[3k+r] F[3k+c]) * volume, i.e. volume * P F^T */
static void OR_NAME(p_ft)(R *PF, const R *P, const R *F, R volume) {
  for (int c = 0; c != 3; ++c)
    for (int r = 0; r != 3; ++r)
      PF[3 * c + r] = (P[r] * F[c] + P[3 + r] * F[3 + c] + P[6 + r] * F[6 + c]) * volume;
}

/* ConstitutiveModel_Vol_dP.hpp:10-46 */
static void OR_NAME(stress_fc)(R volume, R mu, R lambda, const R *F, R *PF) {
  R U[9], S[3], V[9], P[9];
  OR_SVD(F, U, S, V);
  R J = S[0] * S[1] * S[2];
  R scaled_mu = (R)2 * mu;
  R scaled_lambda = lambda * (J - (R)1);
  R Ph[3];
  Ph[0] = scaled_mu * (S[0] - (R)1) + scaled_lambda * (S[1] * S[2]);
  Ph[1] = scaled_mu * (S[1] - (R)1) + scaled_lambda * (S[0] * S[2]);
  Ph[2] = scaled_mu * (S[2] - (R)1) + scaled_lambda * (S[0] * S[1]);
  for (int c = 0; c != 3; ++c)
    for (int r = 0; r != 3; ++r)
      P[3 * c + r] = Ph[0] * U[r] * V[c] + Ph[1] * U[3 + r] * V[3 + c] +
                     Ph[2] * U[6 + r] * V[6 + c];
  OR_NAME(p_ft)(PF, P, F, volume);
}

/* ConstitutiveModel_Vol_dP.hpp:241-325 (F projected in place, logJp updated) */
static void OR_NAME(stress_sand)(R volume, R mu, R lambda, R cohesion, R beta,
                                 R yieldSurface, int volCorrection, R *logJp, R *F, R *PF) {
  R U[9], S[3], V[9];
  OR_SVD(F, U, S, V);
  R scaled_mu = (R)2 * mu;
  R epsilon[3], New_S[3] = {0, 0, 0}, New_F[9];
  for (int i = 0; i != 3; ++i) {
    R abs_S = S[i] > 0 ? S[i] : -S[i];
    /* `abs_S > 1e-4 ? abs_S : 1e-4` compares against the double literal */
    abs_S = ((double)abs_S > 1e-4) ? abs_S : (R)1e-4;
    epsilon[i] = R_LOG(abs_S) - cohesion;
  }
  R sum_epsilon = epsilon[0] + epsilon[1] + epsilon[2];
  R trace_epsilon = sum_epsilon + *logJp;
  R epsilon_hat[3];
  for (int i = 0; i != 3; ++i) epsilon_hat[i] = epsilon[i] - (trace_epsilon / (R)3);
  R epsilon_hat_norm = R_SQRT(epsilon_hat[0] * epsilon_hat[0] + epsilon_hat[1] * epsilon_hat[1] +
                              epsilon_hat[2] * epsilon_hat[2]);
  if (trace_epsilon >= (R)0) {
    New_S[0] = New_S[1] = New_S[2] = R_EXP(cohesion);
    OR_NAME(mat_diag_matT)(New_F, U, New_S, V);
    for (int i = 0; i != 9; ++i) F[i] = New_F[i];
    if (volCorrection) *logJp = beta * sum_epsilon + *logJp;
  } else if (mu != 0) {
    *logJp = 0;
    R delta_gamma = epsilon_hat_norm +
                    ((R)3 * lambda + scaled_mu) / scaled_mu * trace_epsilon * yieldSurface;
    R H[3];
    if (delta_gamma <= 0) {
      for (int i = 0; i != 3; ++i) H[i] = epsilon[i] + cohesion;
    } else {
      for (int i = 0; i != 3; ++i)
        H[i] = epsilon[i] - (delta_gamma / epsilon_hat_norm) * epsilon_hat[i] + cohesion;
    }
    for (int i = 0; i != 3; ++i) New_S[i] = R_EXP(H[i]);
    OR_NAME(mat_diag_matT)(New_F, U, New_S, V);
    for (int i = 0; i != 9; ++i) F[i] = New_F[i];
  }
  R New_S_log[3] = {R_LOG(New_S[0]), R_LOG(New_S[1]), R_LOG(New_S[2])};
  R trace_log_S = New_S_log[0] + New_S_log[1] + New_S_log[2];
  R P_hat[3], P[9];
  for (int i = 0; i != 3; ++i)
    P_hat[i] = (scaled_mu * New_S_log[i] + lambda * trace_log_S) / New_S[i];
  OR_NAME(mat_diag_matT)(P, U, P_hat, V);
  OR_NAME(p_ft)(PF, P, F, volume);
}

/* Snow: SnowPlasticity::do_project_sigma (SnowPlasticity.hpp:24-32) on the singular values
 * of the trial F, committed to F = U diag(S_clamped) V^T; the plastic volume ratio is
 * accumulated, Jp <- Jp * prod(S) / max(prod(S_clamped), 1e-6) (the reference recomputes
 * it from the current step only, which equals this when Jp starts at 1 each step); then
 * fixed-corotated stress with mu, lambda scaled by exp(hardening * (1 - Jp)). */
static void OR_NAME(stress_snow)(R volume, R mu, R lambda, R hardening, R theta_c,
                                 R theta_s, R *Jp, R *F, R *PF) {
  R U[9], S[3], V[9], Sc[3], Fe[9];
  OR_SVD(F, U, S, V);
  R J = S[0] * S[1] * S[2];
  for (int d = 0; d != 3; ++d) {
    R s = S[d] < (R)1 + theta_s ? S[d] : (R)1 + theta_s;
    Sc[d] = s > (R)1 - theta_c ? s : (R)1 - theta_c;
  }
  R Jc = Sc[0] * Sc[1] * Sc[2];
  R jp = *Jp * (J / (Jc > (R)1e-6 ? Jc : (R)1e-6));
  *Jp = jp;
  R e = R_EXP(hardening * ((R)1 - jp));
  OR_NAME(mat_diag_matT)(Fe, U, Sc, V);
  for (int i = 0; i != 9; ++i) F[i] = Fe[i];
  OR_NAME(stress_fc)(volume, mu * e, lambda * e, F, PF);
}

typedef struct {
  int model, mode, wall_type, wall_cells, vc;
  R dx, dt, g[3], E, nu, volume, fa, coh, beta, ys, hard, tc, ts, mu, lam;
} OR_NAME(cfg);

static void OR_NAME(make_cfg)(const oracle_params *p, OR_NAME(cfg) * c) {
  c->model = p->model;
  c->mode = p->mode;
  c->wall_type = p->wall_type;
  c->wall_cells = p->wall_cells;
  c->vc = p->volume_correction;
  c->dx = (R)p->dx;
  c->dt = (R)p->dt;
  c->g[0] = (R)p->gx;
  c->g[1] = (R)p->gy;
  c->g[2] = (R)p->gz;
  c->E = (R)p->E;
  c->nu = (R)p->nu;
  c->volume = (R)p->volume;
  c->fa = (R)p->friction_deg;
  c->coh = (R)p->cohesion;
  c->beta = (R)p->beta;
  c->hard = (R)p->hardening;
  c->tc = (R)p->theta_c;
  c->ts = (R)p->theta_s;
  {
    /* DruckerPragerConfig::yieldSurface (ConstitutiveModel.hpp:752) */
    R sin_phi = (R)sin((double)p->friction_deg / 180.0 * 3.14159265358979323846);
    c->ys = (R)0.816496580927726 * (R)2 * sin_phi / ((R)3 - sin_phi);
    if (sizeof(R) == sizeof(float))
      c->ys = (R)(0.816496580927726f * 2.f * (float)sin_phi / (3.f - (float)sin_phi));
  }
  OR_NAME(lame)(c->E, c->nu, &c->mu, &c->lam);
}

/* Stress of one particle; projects F / updates the plastic variable as the model does. */
static void OR_NAME(stress)(const OR_NAME(cfg) * c, R *F, R *plastic, R *PF) {
  if (c->model == ORACLE_FC)
    OR_NAME(stress_fc)(c->volume, c->mu, c->lam, F, PF);
  else if (c->model == ORACLE_DP)
    OR_NAME(stress_sand)(c->volume, c->mu, c->lam, c->coh, c->beta, c->ys, c->vc, plastic, F, PF);
  else
    OR_NAME(stress_snow)(c->volume, c->mu, c->lam, c->hard, c->tc, c->ts, plastic, F, PF);
}

void OR_NAME(oracle_stress)(const oracle_params *p, R *F, R *plastic, R *PF) {
  OR_NAME(cfg) c;
  OR_NAME(make_cfg)(p, &c);
  OR_NAME(stress)(&c, F, plastic, PF);
}

/* ---- colliders: AnalyticLevelSet signed distances and normals (AnalyticLevelSet.h) and
 * Collider::resolveCollision (Collider.h:80-110), each vector operation in the order of
 * math/VecInterface.hpp (dot/length accumulate from 0 in index order; a matrix-vector product
 * accumulates each row from 0); lengths use the C library square root, as zs::sqrt does on
 * the host (ZpcMathUtils.hpp:760-770) */
static R OR_NAME(col_len)(const R *v) {
  R l2 = 0;
  for (int i = 0; i != 3; ++i) l2 += v[i] * v[i];
  return R_STDSQRT(l2);
}

static R OR_NAME(col_sdf)(const oracle_collider *c, const R *X) {
  if (c->shape == 0) {
    R r = 0;
    for (int i = 0; i != 3; ++i) r += (R)c->b[i] * (X[i] - (R)c->a[i]);
    return r;
  }
  if (c->shape == 1) {
    R p[3], mx;
    for (int i = 0; i != 3; ++i) {
      R center = ((R)c->a[i] + (R)c->b[i]) / (R)2;
      R d = X[i] - center;
      p[i] = (d > 0 ? d : -d) - ((R)c->b[i] - (R)c->a[i]) / (R)2;
    }
    mx = p[0];
    for (int i = 1; i != 3; ++i)
      if (p[i] > mx) mx = p[i];
    for (int i = 0; i != 3; ++i)
      if (p[i] < 0) p[i] = 0;
    return (mx < 0 ? mx : (R)0) + OR_NAME(col_len)(p);
  }
  if (c->shape == 2) {
    R d[3];
    for (int i = 0; i != 3; ++i) d[i] = X[i] - (R)c->a[i];
    return OR_NAME(col_len)(d) - (R)c->b[0];
  }
  {
    const int ax = c->axis;
    R dr[2], l2 = 0;
    for (int k = 0, i = 0; k != 3; ++k)
      if (k != ax) dr[i++] = X[k] - (R)c->a[k];
    for (int i = 0; i != 2; ++i) l2 += dr[i] * dr[i];
    const R dis_r = R_STDSQRT(l2), radius = (R)c->b[0], length = (R)c->b[1], bd = (R)c->a[ax];
    const int outside = dis_r > radius;
    if (X[ax] < bd) {
      R dis_l = bd - X[ax];
      return outside ? R_STDSQRT((dis_r - radius) * (dis_r - radius) + dis_l * dis_l) : dis_l;
    } else if (X[ax] > bd + length) {
      R dis_l = X[ax] - (bd + length);
      return outside ? R_STDSQRT((dis_r - radius) * (dis_r - radius) + dis_l * dis_l) : dis_l;
    } else {
      if (outside) return dis_r - radius;
      R top = bd + length - X[ax], bot = X[ax] - bd;
      R dis_l = top < bot ? top : bot;
      R rr = radius - dis_r;
      return -(dis_l < rr ? dis_l : rr);
    }
  }
}

static void OR_NAME(col_normal)(const oracle_collider *c, const R *X, R *n) {
  if (c->shape == 0) {
    for (int i = 0; i != 3; ++i) n[i] = (R)c->b[i];
    return;
  }
  if (c->shape == 2) {
    R o[3], l2 = 0;
    for (int i = 0; i != 3; ++i) o[i] = X[i] - (R)c->a[i];
    for (int i = 0; i != 3; ++i) l2 += o[i] * o[i];
    if (l2 < (R)1e-7) {
      n[0] = n[1] = n[2] = 0;
      return;
    }
    R len = OR_NAME(col_len)(o);
    for (int i = 0; i != 3; ++i) n[i] = o[i] / len;
    return;
  }
  {
    const R eps = (R)1e-6;
    R diff[3];
    for (int i = 0; i != 3; ++i) {
      R v1[3] = {X[0], X[1], X[2]}, v2[3] = {X[0], X[1], X[2]};
      v1[i] = X[i] + eps;
      v2[i] = X[i] - eps;
      diff[i] = (OR_NAME(col_sdf)(c, v1) - OR_NAME(col_sdf)(c, v2)) / (eps + eps);
    }
    R len = OR_NAME(col_len)(diff);
    for (int i = 0; i != 3; ++i) n[i] = diff[i] / len;
  }
}

static void OR_NAME(col_resolve)(const oracle_collider *c, const R *x, R *v) {
  R xb[3], X[3];
  for (int i = 0; i != 3; ++i) xb[i] = x[i] - (R)c->t[i];
  const R one_over_s = (R)1 / (R)c->s;
  for (int i = 0; i != 3; ++i) {
    R r = 0;
    for (int j = 0; j != 3; ++j) r += (R)c->rot[3 * j + i] * xb[j];
    X[i] = r * one_over_s;
  }
  if (!(OR_NAME(col_sdf)(c, X) < -(R)0)) return;
  R vo[3], cr[3];
  cr[0] = (R)c->omega[1] * xb[2] - (R)c->omega[2] * xb[1];
  cr[1] = (R)c->omega[2] * xb[0] - (R)c->omega[0] * xb[2];
  cr[2] = (R)c->omega[0] * xb[1] - (R)c->omega[1] * xb[0];
  const R ds = (R)c->dsdt * one_over_s;
  for (int i = 0; i != 3; ++i) {
    R mv = 0;  /* R s times the material velocity of an analytic level set (zero) */
    for (int j = 0; j != 3; ++j) mv += ((R)c->rot[3 * i + j] * (R)c->s) * (R)0;
    vo[i] = ((cr[i] + ds * xb[i]) + mv) + (R)c->dtdt[i];
  }
  if (c->type == 0) {
    for (int i = 0; i != 3; ++i) v[i] = vo[i];
    return;
  }
  for (int i = 0; i != 3; ++i) v[i] -= vo[i];
  R nX[3], n[3], proj = 0;
  OR_NAME(col_normal)(c, X, nX);
  for (int i = 0; i != 3; ++i) {
    R r = 0;
    for (int j = 0; j != 3; ++j) r += (R)c->rot[3 * i + j] * nX[j];
    n[i] = r;
  }
  for (int i = 0; i != 3; ++i) proj += n[i] * v[i];
  if ((c->type == 2 && proj < 0) || c->type == 1)
    for (int i = 0; i != 3; ++i) v[i] -= proj * n[i];
  for (int i = 0; i != 3; ++i) v[i] += vo[i];
}

/* ---- sparse level-set boundary: value_or over the blocks (a linear search of the keys; the
 * reference queries its bht), the linear arena with base_node<0> = floor and xlerp with
 * linear_interop(a, b, t) = a + (b - a) t */
static R OR_NAME(ls_node)(const oracle_levelset *L, int32_t cx, int32_t cy, int32_t cz) {
  const int32_t lx = cx & 7, ly = cy & 7, lz = cz & 7;
  const int32_t bx = cx - lx, by = cy - ly, bz = cz - lz;
  for (int b = 0; b != L->nblocks; ++b)
    if (L->keys[3 * b] == bx && L->keys[3 * b + 1] == by && L->keys[3 * b + 2] == bz)
      return (R)L->sdf[(size_t)b * 512 + ((lx << 6) | (ly << 3) | lz)];
  return (R)L->background;
}

static R OR_NAME(ls_lerp)(R t, R a, R b) { return a + (b - a) * t; }

static R OR_NAME(ls_sdf)(const oracle_levelset *L, const R *x) {
  R a[3], b[3], X[3], d[3], p[2][2][2];
  int32_t c[3];
  for (int i = 0; i != 3; ++i) a[i] = x[i] - (R)L->t[i];
  for (int j = 0; j != 3; ++j) {
    R r = 0;
    for (int i = 0; i != 3; ++i) r += (R)L->rinv[3 * i + j] * a[i];
    b[j] = r;
  }
  for (int j = 0; j != 3; ++j) {
    R r = 0;
    for (int i = 0; i != 3; ++i) r += (R)L->sinv[3 * i + j] * b[i];
    X[j] = r;
  }
  for (int k = 0; k != 3; ++k) {
    c[k] = (int32_t)R_FLOOR(X[k]);
    d[k] = X[k] - (R)c[k];
  }
  for (int i = 0; i != 2; ++i)
    for (int j = 0; j != 2; ++j)
      for (int k = 0; k != 2; ++k) p[i][j][k] = OR_NAME(ls_node)(L, c[0] + i, c[1] + j, c[2] + k);
  return OR_NAME(ls_lerp)(
      d[0],
      OR_NAME(ls_lerp)(d[1], OR_NAME(ls_lerp)(d[2], p[0][0][0], p[0][0][1]), OR_NAME(ls_lerp)(d[2], p[0][1][0], p[0][1][1])),
      OR_NAME(ls_lerp)(d[1], OR_NAME(ls_lerp)(d[2], p[1][0][0], p[1][0][1]), OR_NAME(ls_lerp)(d[2], p[1][1][0], p[1][1][1])));
}

/* Collider{levelset, type}.resolveCollision with the identity placement: the collider velocity
 * is zero (the level set has no material-velocity channel) */
static void OR_NAME(ls_resolve)(const oracle_levelset *L, const R *x, R *v) {
  if (!(OR_NAME(ls_sdf)(L, x) < -(R)0)) return;
  if (L->type == 0) {
    for (int i = 0; i != 3; ++i) v[i] = 0;
    return;
  }
  const R eps = (R)1e-6;
  R n[3], proj = 0;
  for (int i = 0; i != 3; ++i) {
    R v1[3] = {x[0], x[1], x[2]}, v2[3] = {x[0], x[1], x[2]};
    v1[i] = x[i] + eps;
    v2[i] = x[i] - eps;
    n[i] = (OR_NAME(ls_sdf)(L, v1) - OR_NAME(ls_sdf)(L, v2)) / (eps + eps);
  }
  const R len = OR_NAME(col_len)(n);
  for (int i = 0; i != 3; ++i) n[i] = n[i] / len;
  for (int i = 0; i != 3; ++i) proj += n[i] * v[i];
  if ((L->type == 2 && proj < 0) || L->type == 1)
    for (int i = 0; i != 3; ++i) v[i] -= proj * n[i];
}

/* quadratic B-spline stencil (Utils.hpp:30-70, InterpolationKernel.hpp:51-57, :93-130) */
typedef struct {
  int corner[3];
  R w[3][3];
  R localPos[3]; /* (X - corner) * dx */
} OR_NAME(arena);

static void OR_NAME(make_arena)(OR_NAME(arena) * a, R dx, const R *pos) {
  for (int d = 0; d != 3; ++d) {
    R X = pos[d] / dx;
    a->corner[d] = (int)R_FLOOR(X - (R)0.5);
    R lp = X - (R)a->corner[d];
    R d0 = lp - (R)(int)R_FLOOR(lp - (R)0.5);
    a->w[d][0] = (R)0.5 * ((R)1.5 - d0) * ((R)1.5 - d0);
    R d1 = d0 - (R)1.0;
    a->w[d][1] = (R)0.75 - d1 * d1;
    R zz = (R)0.5 + d1;
    a->w[d][2] = (R)0.5 * zz * zz;
    a->localPos[d] = lp * dx;
  }
}

static int OR_NAME(block_of)(const R *x, R dxinv, int32_t *out) {
  for (int d = 0; d != 3; ++d) {
    R v = x[d] * dxinv + (R)0.5;
    if (!(v > -1e9 && v < 1e9)) return 1;
    int32_t c = (int32_t)R_FLOOR(v) - 2;
    out[d] = (c + (c < 0 ? -7 : 0)) / 8;
  }
  return 0;
}

int OR_NAME(oracle_run)(const oracle_params *p, int n, const R *m, R *x, R *v, R *C, R *F,
                        R *plastic, int nsteps, int cap_blocks, int *out_nblocks,
                        int *out_keys, R *out_grid) {
  OR_NAME(cfg) cfg;
  OR_NAME(make_cfg)(p, &cfg);
  const R dx = cfg.dx, dt = cfg.dt;
  const R dx_inv = (R)1 / dx;
  const R D_inv = (R)4 * dx_inv * dx_inv;
  oracle_table t;
  if (oracle_table_init(&t, p->table_expected)) return 3;
  R *grid = NULL;
  size_t grid_blocks = 0;
  R *tau = NULL;
  int status = 0;
  if (cfg.mode == ORACLE_MODE_COMMITTED) {
    /* stress of the initial state, computed as the end of a G2P would */
    tau = (R *)malloc(sizeof(R) * 9 * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i != n; ++i) OR_NAME(stress)(&cfg, &F[9 * i], &plastic[i], &tau[9 * i]);
  }
  for (int step = 0; step != nsteps && !status; ++step) {
    /* 1. activation (SparsityOp.hpp:58-112) and canonical order */
    oracle_table_clear(&t);
    for (int i = 0; i != n && !status; ++i) {
      int32_t b[3];
      if (OR_NAME(block_of)(&x[3 * i], dx_inv, b)) status = 4;
      else if (oracle_table_insert(&t, b, -1) < 0) status = 2;
    }
    const int npb = t.count;
    for (int i = 0; i != npb && !status; ++i) {
      int32_t k[3] = {t.active[3 * i], t.active[3 * i + 1], t.active[3 * i + 2]};
      for (int a = 0; a != 2; ++a)
        for (int b = 0; b != 2; ++b)
          for (int c = 0; c != 2; ++c) {
            int32_t nk[3] = {k[0] + a, k[1] + b, k[2] + c};
            if (oracle_table_insert(&t, nk, -1) < 0) status = 2;
          }
    }
    if (status) break;
    if (t.count >= t.size - 20) {
      status = 2;
      break;
    }
    oracle_table_canonicalize(&t);
    const int nb = t.count;
    if ((size_t)nb > grid_blocks) {
      free(grid);
      grid_blocks = (size_t)nb;
      grid = (R *)malloc(sizeof(R) * 7 * 512 * grid_blocks);
    }
    memset(grid, 0, sizeof(R) * 7 * 512 * (size_t)nb);

    /* 2. P2G (P2G.hpp:45-127) */
    for (int i = 0; i != n; ++i) {
      const R *xp = &x[3 * i], *vp = &v[3 * i], *Cp = &C[9 * i];
      const R mass = m[i];
      R contrib[9];
      if (cfg.mode == ORACLE_MODE_REFERENCE) {
        R Fl[9];
        for (int k = 0; k != 9; ++k) Fl[k] = F[9 * i + k];
        OR_NAME(stress)(&cfg, Fl, &plastic[i], contrib);
      } else {
        for (int k = 0; k != 9; ++k) contrib[k] = tau[9 * i + k];
      }
      for (int k = 0; k != 9; ++k) contrib[k] = contrib[k] * -dt * D_inv;
      OR_NAME(arena) a;
      OR_NAME(make_arena)(&a, dx, xp);
      for (int ii = 0; ii != 3; ++ii)
        for (int jj = 0; jj != 3; ++jj)
          for (int kk = 0; kk != 3; ++kk) {
            int32_t coord[3] = {a.corner[0] + ii, a.corner[1] + jj, a.corner[2] + kk};
            int32_t loc[3], bk[3];
            for (int d = 0; d != 3; ++d) {
              loc[d] = coord[d] & 7;
              bk[d] = (coord[d] - loc[d]) / 8;
            }
            int32_t blk = oracle_table_query(&t, bk);
            if (blk < 0) {
              status = 5;
              continue;
            }
            R xixp[3] = {(R)ii * dx - a.localPos[0], (R)jj * dx - a.localPos[1],
                         (R)kk * dx - a.localPos[2]};
            R W = a.w[0][ii] * a.w[1][jj] * a.w[2][kk];
            int cell = (loc[0] << 6) | (loc[1] << 3) | loc[2];
            R *g = &grid[(size_t)blk * 7 * 512];
            g[0 * 512 + cell] += mass * W;
            for (int d = 0; d != 3; ++d) {
              g[(1 + d) * 512 + cell] +=
                  W * mass * (vp[d] + (Cp[d] * xixp[0] + Cp[3 + d] * xixp[1] + Cp[6 + d] * xixp[2]));
              g[(4 + d) * 512 + cell] +=
                  (contrib[d] * xixp[0] + contrib[3 + d] * xixp[1] + contrib[6 + d] * xixp[2]) * W;
            }
          }
    }
    if (status) break;

    /* 3. grid velocity, v = (mv + rhs) / m + g dt (restated), then walls */
    const R lo = (R)cfg.wall_cells * dx, hi = (R)1 - (R)cfg.wall_cells * dx;
    for (int b = 0; b != nb; ++b) {
      R *g = &grid[(size_t)b * 7 * 512];
      const int32_t *key = &t.active[3 * b];
      for (int cell = 0; cell != 512; ++cell) {
        R mass = g[cell];
        if (mass != 0) {
          mass = (R)1 / mass;
          R vel[3];
          for (int d = 0; d != 3; ++d)
            vel[d] = (g[(1 + d) * 512 + cell] + g[(4 + d) * 512 + cell]) * mass + cfg.g[d] * dt;
          for (int d = 0; d != 3; ++d) g[(1 + d) * 512 + cell] = vel[d];
        }
      }
      if (cfg.wall_type == ORACLE_WALL_NONE) continue;
      /* ApplyBoundaryConditionOnGridBlocks once per wall, walls x-,x+,y-,y+,z-,z+ */
      for (int w = 0; w != 6; ++w) {
        const int axis = w / 2;
        const R sgn = (w & 1) ? (R)-1 : (R)1;
        const R origin = (w & 1) ? hi : lo;
        for (int cell = 0; cell != 512; ++cell) {
          if (!(g[cell] > 0)) continue;
          const int cc[3] = {cell >> 6, (cell >> 3) & 7, cell & 7};
          R pos = ((R)key[axis] * (R)8 + (R)cc[axis]) * dx;
          R sd = sgn * (pos - origin);
          if (!(sd < 0)) continue;
          if (cfg.wall_type == ORACLE_WALL_STICKY) {
            for (int d = 0; d != 3; ++d) g[(1 + d) * 512 + cell] = 0;
          } else {
            R proj = sgn * g[(1 + axis) * 512 + cell];
            if (cfg.wall_type == ORACLE_WALL_SLIP || proj < 0)
              g[(1 + axis) * 512 + cell] = g[(1 + axis) * 512 + cell] - proj * sgn;
          }
        }
      }
    }
    /* the colliders after the walls, each over every node with positive mass */
    for (int k = 0; k != p->ncolliders; ++k)
      for (int b = 0; b != nb; ++b) {
        R *g = &grid[(size_t)b * 7 * 512];
        const int32_t *key = &t.active[3 * b];
        for (int cell = 0; cell != 512; ++cell) {
          if (!(g[cell] > 0)) continue;
          const int cc[3] = {cell >> 6, (cell >> 3) & 7, cell & 7};
          R pos[3], vel[3];
          for (int d = 0; d != 3; ++d) {
            pos[d] = ((R)key[d] * (R)8 + (R)cc[d]) * dx;
            vel[d] = g[(1 + d) * 512 + cell];
          }
          OR_NAME(col_resolve)(&p->colliders[k], pos, vel);
          for (int d = 0; d != 3; ++d) g[(1 + d) * 512 + cell] = vel[d];
        }
      }
    /* then the sparse level sets */
    for (int k = 0; k != p->nlevelsets; ++k)
      for (int b = 0; b != nb; ++b) {
        R *g = &grid[(size_t)b * 7 * 512];
        const int32_t *key = &t.active[3 * b];
        for (int cell = 0; cell != 512; ++cell) {
          if (!(g[cell] > 0)) continue;
          const int cc[3] = {cell >> 6, (cell >> 3) & 7, cell & 7};
          R pos[3], vel[3];
          for (int d = 0; d != 3; ++d) {
            pos[d] = ((R)key[d] * (R)8 + (R)cc[d]) * dx;
            vel[d] = g[(1 + d) * 512 + cell];
          }
          OR_NAME(ls_resolve)(&p->levelsets[k], pos, vel);
          for (int d = 0; d != 3; ++d) g[(1 + d) * 512 + cell] = vel[d];
        }
      }

    /* 4. G2P (G2P.hpp:43-84), then in committed mode the constitutive update */
    for (int i = 0; i != n; ++i) {
      R *xp = &x[3 * i], *vp = &v[3 * i], *Cp = &C[9 * i], *Fp = &F[9 * i];
      R vel[3] = {0, 0, 0}, Cn[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      OR_NAME(arena) a;
      OR_NAME(make_arena)(&a, dx, xp);
      for (int ii = 0; ii != 3; ++ii)
        for (int jj = 0; jj != 3; ++jj)
          for (int kk = 0; kk != 3; ++kk) {
            int32_t coord[3] = {a.corner[0] + ii, a.corner[1] + jj, a.corner[2] + kk};
            int32_t loc[3], bk[3];
            for (int d = 0; d != 3; ++d) {
              loc[d] = coord[d] & 7;
              bk[d] = (coord[d] - loc[d]) / 8;
            }
            int32_t blk = oracle_table_query(&t, bk);
            R xixp[3] = {(R)ii * dx - a.localPos[0], (R)jj * dx - a.localPos[1],
                         (R)kk * dx - a.localPos[2]};
            R W = a.w[0][ii] * a.w[1][jj] * a.w[2][kk];
            int cell = (loc[0] << 6) | (loc[1] << 3) | loc[2];
            const R *g = &grid[(size_t)blk * 7 * 512];
            R vi[3] = {g[1 * 512 + cell], g[2 * 512 + cell], g[3 * 512 + cell]};
            for (int d = 0; d != 3; ++d) vel[d] += vi[d] * W;
            for (int d = 0; d != 9; ++d) Cn[d] += W * vi[d % 3] * xixp[d / 3] * D_inv;
          }
      for (int d = 0; d != 3; ++d) xp[d] += vel[d] * dt;
      {
        R tmp[9], Fn[9];
        for (int d = 0; d != 9; ++d) tmp[d] = Cn[d] * dt + ((d & 0x3) ? (R)0 : (R)1);
        for (int c = 0; c != 3; ++c)
          for (int r = 0; r != 3; ++r)
            Fn[3 * c + r] = tmp[r] * Fp[3 * c] + tmp[3 + r] * Fp[3 * c + 1] + tmp[6 + r] * Fp[3 * c + 2];
        for (int d = 0; d != 9; ++d) Fp[d] = Fn[d];
      }
      for (int d = 0; d != 3; ++d) vp[d] = vel[d];
      for (int d = 0; d != 9; ++d) Cp[d] = Cn[d];
      if (cfg.mode == ORACLE_MODE_COMMITTED) OR_NAME(stress)(&cfg, Fp, &plastic[i], &tau[9 * i]);
    }
  }
  if (!status) {
    const int nb = t.count;
    if (out_nblocks) *out_nblocks = nb;
    if (out_keys) {
      if (nb > cap_blocks) status = 1;
      else
        for (int b = 0; b != nb; ++b) {
          for (int d = 0; d != 3; ++d) out_keys[3 * b + d] = t.active[3 * b + d];
          for (int ch = 0; ch != 4; ++ch)
            for (int cell = 0; cell != 512; ++cell)
              out_grid[((size_t)b * 4 + ch) * 512 + cell] = grid[((size_t)b * 7 + ch) * 512 + cell];
        }
    }
  }
  free(grid);
  free(tau);
  oracle_table_free(&t);
  return status;
}

/* G2P2GTransfer (simulation/transfer/G2P2G.hpp:49-142), the implicit force operator: per
 * particle, C from the velocity field vin, the trial F = (I + dt C) F (MatrixUtils.h:136-146),
 * its stress on a copy of the state (:103-123; nothing is written back), then
 * fout[node] += W (D_inv V0 P F^T)(x_i - x_p) (:125-140).  vin and fout are node-major over
 * the given blocks, [(block*512 + cell)*3 + d], the layout of a dof_view<space, 3> over a
 * Vector (types/View.h:77-168); block b of keys gets index b.  fout is zeroed first.  Returns
 * 0, 2 when the table is full, 5 when a stencil node falls outside the blocks. */
int OR_NAME(oracle_g2p2g)(const oracle_params *p, int n, const R *x, const R *F, const R *plastic,
                          int nb, const int32_t *keys, const R *vin, R *fout) {
  OR_NAME(cfg) cfg;
  OR_NAME(make_cfg)(p, &cfg);
  const R dx = cfg.dx, dt = cfg.dt;
  const R dx_inv = (R)1 / dx;
  const R D_inv = (R)4 * dx_inv * dx_inv;
  oracle_table t;
  if (oracle_table_init(&t, p->table_expected > nb ? p->table_expected : nb)) return 3;
  int status = 0;
  for (int b = 0; b != nb && !status; ++b)
    if (oracle_table_insert(&t, &keys[3 * b], b) < 0) status = 2;
  memset(fout, 0, sizeof(R) * 1536 * (size_t)(nb > 0 ? nb : 0));
  for (int i = 0; i != n && !status; ++i) {
    const R *xp = &x[3 * i];
    R Cn[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, contrib[9];
    OR_NAME(arena) a;
    OR_NAME(make_arena)(&a, dx, xp);
    int32_t node[27];
    for (int ii = 0; ii != 3; ++ii)
      for (int jj = 0; jj != 3; ++jj)
        for (int kk = 0; kk != 3; ++kk) {
          int32_t coord[3] = {a.corner[0] + ii, a.corner[1] + jj, a.corner[2] + kk};
          int32_t loc[3], bk[3];
          for (int d = 0; d != 3; ++d) {
            loc[d] = coord[d] & 7;
            bk[d] = (coord[d] - loc[d]) / 8;
          }
          const int32_t blk = oracle_table_query(&t, bk);
          const int q = (ii * 3 + jj) * 3 + kk;
          if (blk < 0) {
            status = 5;
            node[q] = -1;
            continue;
          }
          node[q] = blk * 512 + ((loc[0] << 6) | (loc[1] << 3) | loc[2]);
          R xixp[3] = {(R)ii * dx - a.localPos[0], (R)jj * dx - a.localPos[1],
                       (R)kk * dx - a.localPos[2]};
          R W = a.w[0][ii] * a.w[1][jj] * a.w[2][kk];
          const R *vi = &vin[(size_t)node[q] * 3];
          for (int d = 0; d != 9; ++d) Cn[d] += W * vi[d % 3] * xixp[d / 3] * D_inv;
        }
    if (status) break;
    R Fl[9], pl = plastic ? plastic[i] : (R)0;
    {
      R tmp[9];
      const R *Fp = &F[9 * i];
      for (int d = 0; d != 9; ++d) tmp[d] = Cn[d] * dt + ((d & 0x3) ? (R)0 : (R)1);
      for (int c = 0; c != 3; ++c)
        for (int r = 0; r != 3; ++r)
          Fl[3 * c + r] = tmp[r] * Fp[3 * c] + tmp[3 + r] * Fp[3 * c + 1] + tmp[6 + r] * Fp[3 * c + 2];
    }
    OR_NAME(stress)(&cfg, Fl, &pl, contrib);
    for (int d = 0; d != 9; ++d) contrib[d] = contrib[d] * D_inv;
    for (int ii = 0; ii != 3; ++ii)
      for (int jj = 0; jj != 3; ++jj)
        for (int kk = 0; kk != 3; ++kk) {
          const int q = (ii * 3 + jj) * 3 + kk;
          R xixp[3] = {(R)ii * dx - a.localPos[0], (R)jj * dx - a.localPos[1],
                       (R)kk * dx - a.localPos[2]};
          R W = a.w[0][ii] * a.w[1][jj] * a.w[2][kk];
          R *fi = &fout[(size_t)node[q] * 3];
          for (int d = 0; d != 3; ++d)
            fi[d] += W * (contrib[d] * xixp[0] + contrib[3 + d] * xixp[1] + contrib[6 + d] * xixp[2]);
        }
  }
  oracle_table_free(&t);
  return status;
}


/* ---- the cell-centric transfer pair: P2C2GTransfer (simulation/transfer/P2C2G.hpp:27-189)
 * and G2C2PTransfer with PreG2C2PTransfer / PostG2C2PTransfer (G2C2P.hpp:36-278), the
 * fixed-corotated branch, on the index buckets of simulation/particle/Query.tpp:8-58 (one
 * bucket per cell coordinate floor(x / dx + 0.5), particles in index order within a bucket,
 * as a sequential SpatiallyDistribute leaves them).  Cells run in block-index then cell order
 * and particles within a bucket in index order, the sequential schedule of the compiled
 * reference; the atomics of the reference are plain additions in that order. */
typedef struct {
  uint64_t key;
  int32_t idx;
} OR_NAME(bucket_entry);

static int OR_NAME(bucket_cmp)(const void *a, const void *b) {
  const OR_NAME(bucket_entry) *x = (const OR_NAME(bucket_entry) *)a, *y = (const OR_NAME(bucket_entry) *)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

static uint64_t OR_NAME(bucket_key)(int32_t bx, int32_t by, int32_t bz) {
  const uint64_t bias = (uint64_t)1 << 20;
  return (((uint64_t)(bx + (int64_t)bias)) << 42) | (((uint64_t)(by + (int64_t)bias)) << 21) |
         (uint64_t)(bz + (int64_t)bias);
}

/* [*first, *last) of the entries of bucket (bx, by, bz) */
static void OR_NAME(bucket_range)(const OR_NAME(bucket_entry) * e, int n, int32_t bx, int32_t by, int32_t bz,
                                  int *first, int *last) {
  const uint64_t k = OR_NAME(bucket_key)(bx, by, bz);
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (e[mid].key < k) lo = mid + 1;
    else hi = mid;
  }
  *first = lo;
  while (lo < n && e[lo].key == k) ++lo;
  *last = lo;
}

/* Dinv of a position component (P2C2G.hpp:87-91, G2C2P.hpp PostG2C2PTransfer): the offset from
 * the nearest node, then 2 / (dx^2 - 2 offset^2) */
static R OR_NAME(cell_dinv)(R pos, R dx, R dx_inv) {
  R X = pos - (R)(int32_t)R_FLOOR(pos * dx_inv + (R)0.5) * dx;
  return (R)2 / (dx * dx - (R)2 * X * X);
}

int OR_NAME(oracle_run_cell)(const oracle_params *p, int n, const R *m, R *x, R *v, R *C, R *F, int nsteps,
                             int cap_blocks, int *out_nblocks, int *out_keys, R *out_grid) {
  OR_NAME(cfg) cfg;
  OR_NAME(make_cfg)(p, &cfg);
  if (cfg.model != ORACLE_FC) return 6;
  const R dx = cfg.dx, dt = cfg.dt;
  const R dx_inv = (R)1 / dx;
  oracle_table t;
  if (oracle_table_init(&t, p->table_expected)) return 3;
  R *grid = NULL;
  size_t grid_blocks = 0;
  int status = 0;
  OR_NAME(bucket_entry) *bk = (OR_NAME(bucket_entry) *)malloc(sizeof(*bk) * (size_t)(n > 0 ? n : 1));
  R *contrib = (R *)malloc(sizeof(R) * 9 * (size_t)(n > 0 ? n : 1));
  for (int step = 0; step != nsteps && !status; ++step) {
    /* activation (SparsityOp.hpp:58-112) and canonical order, as in oracle_run */
    oracle_table_clear(&t);
    for (int i = 0; i != n && !status; ++i) {
      int32_t b[3];
      if (OR_NAME(block_of)(&x[3 * i], dx_inv, b)) status = 4;
      else if (oracle_table_insert(&t, b, -1) < 0) status = 2;
    }
    const int npb = t.count;
    for (int i = 0; i != npb && !status; ++i) {
      int32_t k[3] = {t.active[3 * i], t.active[3 * i + 1], t.active[3 * i + 2]};
      for (int a = 0; a != 2; ++a)
        for (int b = 0; b != 2; ++b)
          for (int c = 0; c != 2; ++c) {
            int32_t nk[3] = {k[0] + a, k[1] + b, k[2] + c};
            if (oracle_table_insert(&t, nk, -1) < 0) status = 2;
          }
    }
    if (status) break;
    if (t.count >= t.size - 20) {
      status = 2;
      break;
    }
    oracle_table_canonicalize(&t);
    const int nb = t.count;
    if ((size_t)nb > grid_blocks) {
      free(grid);
      grid_blocks = (size_t)nb;
      grid = (R *)malloc(sizeof(R) * 4 * 512 * grid_blocks);
    }
    memset(grid, 0, sizeof(R) * 4 * 512 * (size_t)nb);

    /* index buckets (Query.tpp:20-56, ComputeSparsity with blockLen 1, displacement 0.5) */
    for (int i = 0; i != n; ++i) {
      int32_t c[3];
      for (int d = 0; d != 3; ++d) c[d] = (int32_t)R_FLOOR(x[3 * i + d] * dx_inv + (R)0.5);
      bk[i].key = OR_NAME(bucket_key)(c[0], c[1], c[2]);
      bk[i].idx = i;
    }
    qsort(bk, (size_t)n, sizeof(*bk), OR_NAME(bucket_cmp));

    /* the per-particle part of P2C2G (P2C2G.hpp:87-146): contrib = (m B - dt V0 P F^T) Dinv,
     * columns scaled; a function of the particle alone, evaluated once per particle */
    for (int i = 0; i != n; ++i) {
      R Dinv[3], Cs[9], PF[9];
      for (int d = 0; d != 3; ++d) Dinv[d] = OR_NAME(cell_dinv)(x[3 * i + d], dx, dx_inv);
      for (int d = 0; d != 9; ++d) Cs[d] = C[9 * i + d] * Dinv[d / 3];
      OR_NAME(stress_fc)(cfg.volume, cfg.mu, cfg.lam, &F[9 * i], PF);
      for (int d = 0; d != 9; ++d) PF[d] = PF[d] * (Dinv[d / 3] * -dt);
      for (int d = 0; d != 9; ++d) contrib[9 * i + d] = PF[d] + Cs[d] * m[i];
    }

    /* P2C2G over every (block, cell): stage 1 gathers the particles within dx of the cell's
     * center (tent weights), stage 2 adds the cell's sums to its 8 corner nodes (1/8 each) */
    for (int b = 0; b != nb; ++b) {
      const int32_t *key = &t.active[3 * b];
      for (int cell = 0; cell != 512; ++cell) {
        const int32_t coord[3] = {key[0] * 8 + (cell >> 6), key[1] * 8 + ((cell >> 3) & 7), key[2] * 8 + (cell & 7)};
        R posc[3];
        for (int d = 0; d != 3; ++d) posc[d] = ((R)coord[d] + (R)0.5) * dx;
        R m_c = 0, mv_c[3] = {0, 0, 0}, QD[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, QDX[3] = {0, 0, 0};
        for (int a = 0; a != 3; ++a)
          for (int bb = 0; bb != 3; ++bb)
            for (int c = 0; c != 3; ++c) {
              int first, last;
              OR_NAME(bucket_range)(bk, n, coord[0] - 1 + a, coord[1] - 1 + bb, coord[2] - 1 + c, &first, &last);
              for (int e = first; e != last; ++e) {
                const int i = bk[e].idx;
                const R *posp = &x[3 * i];
                int in = 1;
                for (int d = 0; d != 3; ++d)
                  if (R_ABS(posp[d] - posc[d]) > dx) in = 0;
                if (!in) continue;
                const R *q = &contrib[9 * i];
                R Wpc = 1;
                for (int d = 0; d != 3; ++d) Wpc *= ((R)1 - R_ABS((posc[d] - posp[d]) * dx_inv));
                m_c += m[i] * Wpc;
                for (int d = 0; d != 3; ++d) {
                  mv_c[d] += m[i] * v[3 * i + d] * Wpc;
                  QDX[d] += (q[d] * posp[0] + q[3 + d] * posp[1] + q[6 + d] * posp[2]) * Wpc;
                }
                for (int d = 0; d != 9; ++d) QD[d] += q[d] * Wpc;
              }
            }
        for (int a = 0; a != 2; ++a)
          for (int bb = 0; bb != 2; ++bb)
            for (int c = 0; c != 2; ++c) {
              const int32_t ci[3] = {coord[0] + a, coord[1] + bb, coord[2] + c};
              int32_t loc[3], bkey[3];
              R posi[3];
              for (int d = 0; d != 3; ++d) {
                loc[d] = ci[d] & 7;
                bkey[d] = (ci[d] - loc[d]) / 8;
                posi[d] = (R)ci[d] * dx;
              }
              const int32_t blk = oracle_table_query(&t, bkey);
              if (blk < 0) continue;
              const R Wci = (R)0.125;
              const int nc = (loc[0] << 6) | (loc[1] << 3) | loc[2];
              R *g = &grid[(size_t)blk * 4 * 512];
              g[nc] += m_c * Wci;
              for (int d = 0; d != 3; ++d)
                g[(1 + d) * 512 + nc] +=
                    (mv_c[d] + ((QD[d] * posi[0] + QD[3 + d] * posi[1] + QD[6 + d] * posi[2]) - QDX[d])) * Wci;
            }
      }
    }

    /* grid velocity and walls, as in oracle_run (the restated rhs channel is zero here) */
    const R lo = (R)cfg.wall_cells * dx, hi = (R)1 - (R)cfg.wall_cells * dx;
    for (int b = 0; b != nb; ++b) {
      R *g = &grid[(size_t)b * 4 * 512];
      const int32_t *key = &t.active[3 * b];
      for (int cell = 0; cell != 512; ++cell) {
        R mass = g[cell];
        if (mass != 0) {
          mass = (R)1 / mass;
          R vel[3];
          for (int d = 0; d != 3; ++d) vel[d] = (g[(1 + d) * 512 + cell] + (R)0) * mass + cfg.g[d] * dt;
          for (int d = 0; d != 3; ++d) g[(1 + d) * 512 + cell] = vel[d];
        }
      }
      if (cfg.wall_type == ORACLE_WALL_NONE) continue;
      for (int w = 0; w != 6; ++w) {
        const int axis = w / 2;
        const R sgn = (w & 1) ? (R)-1 : (R)1;
        const R origin = (w & 1) ? hi : lo;
        for (int cell = 0; cell != 512; ++cell) {
          if (!(g[cell] > 0)) continue;
          const int cc[3] = {cell >> 6, (cell >> 3) & 7, cell & 7};
          R pos = ((R)key[axis] * (R)8 + (R)cc[axis]) * dx;
          R sd = sgn * (pos - origin);
          if (!(sd < 0)) continue;
          if (cfg.wall_type == ORACLE_WALL_STICKY) {
            for (int d = 0; d != 3; ++d) g[(1 + d) * 512 + cell] = 0;
          } else {
            R proj = sgn * g[(1 + axis) * 512 + cell];
            if (cfg.wall_type == ORACLE_WALL_SLIP || proj < 0)
              g[(1 + axis) * 512 + cell] = g[(1 + axis) * 512 + cell] - proj * sgn;
          }
        }
      }
    }

    /* PreG2C2PTransfer, then G2C2PTransfer over every (block, cell): the cell's mean corner
     * velocity and its moment, added to the particles within dx of the center */
    R *B = C;
    for (int i = 0; i != n; ++i) {
      for (int d = 0; d != 3; ++d) v[3 * i + d] = 0;
      for (int d = 0; d != 9; ++d) B[9 * i + d] = 0;
    }
    for (int b = 0; b != nb; ++b) {
      const int32_t *key = &t.active[3 * b];
      for (int cell = 0; cell != 512; ++cell) {
        const int32_t coord[3] = {key[0] * 8 + (cell >> 6), key[1] * 8 + ((cell >> 3) & 7), key[2] * 8 + (cell & 7)};
        R v_c[3] = {0, 0, 0}, vx_c[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int a = 0; a != 2; ++a)
          for (int bb = 0; bb != 2; ++bb)
            for (int c = 0; c != 2; ++c) {
              const int32_t ci[3] = {coord[0] + a, coord[1] + bb, coord[2] + c};
              int32_t loc[3], bkey[3];
              R posi[3];
              for (int d = 0; d != 3; ++d) {
                loc[d] = ci[d] & 7;
                bkey[d] = (ci[d] - loc[d]) / 8;
                posi[d] = (R)ci[d] * dx;
              }
              const int32_t blk = oracle_table_query(&t, bkey);
              if (blk < 0) continue;
              const R W = (R)0.125;
              const int nc = (loc[0] << 6) | (loc[1] << 3) | loc[2];
              const R *g = &grid[(size_t)blk * 4 * 512];
              const R vi[3] = {g[1 * 512 + nc], g[2 * 512 + nc], g[3 * 512 + nc]};
              for (int d = 0; d != 3; ++d) v_c[d] += vi[d] * W;
              for (int d = 0; d != 9; ++d) vx_c[d] += W * vi[d % 3] * posi[d / 3];
            }
        R posc[3];
        for (int d = 0; d != 3; ++d) posc[d] = ((R)coord[d] + (R)0.5) * dx;
        for (int a = 0; a != 3; ++a)
          for (int bb = 0; bb != 3; ++bb)
            for (int c = 0; c != 3; ++c) {
              int first, last;
              OR_NAME(bucket_range)(bk, n, coord[0] - 1 + a, coord[1] - 1 + bb, coord[2] - 1 + c, &first, &last);
              for (int e = first; e != last; ++e) {
                const int i = bk[e].idx;
                const R *posp = &x[3 * i];
                int in = 1;
                for (int d = 0; d != 3; ++d)
                  if (R_ABS(posp[d] - posc[d]) > dx) in = 0;
                if (!in) continue;
                R W = 1;
                for (int d = 0; d != 3; ++d) {
                  const R xabs = R_ABS((posc[d] - posp[d]) * dx_inv);
                  if (xabs <= (R)1) W *= ((R)1 - xabs);
                  else W *= (R)0;
                }
                for (int d = 0; d != 3; ++d) v[3 * i + d] += v_c[d] * W;
                for (int d = 0; d != 9; ++d) B[9 * i + d] += W * (vx_c[d] - v_c[d % 3] * posp[d / 3]);
              }
            }
      }
    }
    /* PostG2C2PTransfer: F <- (I + dt B Dinv) F, x += v dt; B stays in C */
    for (int i = 0; i != n; ++i) {
      R *xp = &x[3 * i], *Fp = &F[9 * i];
      R Dinv[3], Cs[9], tmp[9], Fn[9];
      for (int d = 0; d != 3; ++d) Dinv[d] = OR_NAME(cell_dinv)(xp[d], dx, dx_inv);
      for (int d = 0; d != 9; ++d) Cs[d] = B[9 * i + d] * Dinv[d / 3];
      for (int d = 0; d != 9; ++d) tmp[d] = Cs[d] * dt + ((d & 0x3) ? (R)0 : (R)1);
      for (int c = 0; c != 3; ++c)
        for (int r = 0; r != 3; ++r)
          Fn[3 * c + r] = tmp[r] * Fp[3 * c] + tmp[3 + r] * Fp[3 * c + 1] + tmp[6 + r] * Fp[3 * c + 2];
      for (int d = 0; d != 9; ++d) Fp[d] = Fn[d];
      for (int d = 0; d != 3; ++d) xp[d] += v[3 * i + d] * dt;
    }
  }
  if (!status) {
    const int nb = t.count;
    if (out_nblocks) *out_nblocks = nb;
    if (out_keys) {
      if (nb > cap_blocks) status = 1;
      else
        for (int b = 0; b != nb; ++b) {
          for (int d = 0; d != 3; ++d) out_keys[3 * b + d] = t.active[3 * b + d];
          memcpy(&out_grid[(size_t)b * 4 * 512], &grid[(size_t)b * 4 * 512], sizeof(R) * 4 * 512);
        }
    }
  }
  free(grid);
  free(bk);
  free(contrib);
  oracle_table_free(&t);
  return status;
}

#undef OR_NAME
#undef OR_CAT
#undef OR_CAT2
