// CPU oracle, part 2: L-BFGS-B v3.0 restated (test infrastructure only).
//
// Follows src/lbfgsb/lbfgsb.f (Byrd, Lu, Nocedal & Zhu 1995; Morales &
// Nocedal 2011 remark): compact limited-memory matrices, generalized Cauchy
// point by breakpoint heap, subspace minimization with the 2011 projection
// step, More-Thuente line search.  The reverse-communication protocol is the
// one setulb exposes: every return asks the caller either for f/g at x
// (TASK_FG) or announces a finished iteration (TASK_NEW_X).  Line numbers in
// the comments refer to lbfgsb.f.  Arrays are column-major like the Fortran
// so the small dense algebra reads the same; variable names follow the paper.
#include "oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

namespace {

const double kBig = 1.0e10;

// Cholesky of the leading nn x nn block of a (lda stride), upper factor R with
// A = R^T R stored in the upper triangle (linpack dpofa, linpack.f:6-80).
int chol_upper(double* a, int lda, int nn) {
  for (int j = 0; j < nn; ++j) {
    double s = 0.0;
    for (int k = 0; k < j; ++k) {
      double t = a[k + j * lda];
      for (int i = 0; i < k; ++i) t -= a[i + k * lda] * a[i + j * lda];
      t /= a[k + k * lda];
      a[k + j * lda] = t;
      s += t * t;
    }
    s = a[j + j * lda] - s;
    if (s <= 0.0) return j + 1;
    a[j + j * lda] = std::sqrt(s);
  }
  return 0;
}

// Triangular solves with an upper factor (linpack dtrsl, linpack.f:81-218):
// trans=true solves R^T x = b (job 11), trans=false solves R x = b (job 01).
int tri_solve(const double* t, int ldt, int nn, double* b, bool trans) {
  for (int i = 0; i < nn; ++i)
    if (t[i + i * ldt] == 0.0) return i + 1;
  if (trans) {
    for (int j = 0; j < nn; ++j) {
      double s = b[j];
      for (int i = 0; i < j; ++i) s -= t[i + j * ldt] * b[i];
      b[j] = s / t[j + j * ldt];
    }
  } else {
    for (int j = nn - 1; j >= 0; --j) {
      b[j] /= t[j + j * ldt];
      const double bj = b[j];
      for (int i = 0; i < j; ++i) b[i] -= bj * t[i + j * ldt];
    }
  }
  return 0;
}

struct Lbfgsb {
  // problem
  int n, m;
  std::vector<double> lo, up;
  std::vector<int> nbd;
  double factr, pgtol;
  // limited-memory matrices (column-major, like ws(n,m), sy(m,m), wn(2m,2m))
  std::vector<double> ws, wy, sy, ss, wt, wn, snd;
  std::vector<double> z, r, d, t, xp, wa;
  std::vector<int> index, iwhere, indx2;
  // scalar state (setulb's isave/dsave/lsave)
  bool prjctd = false, cnstnd = false, boxed = false, updatd = false, wrk = false;
  int col = 0, head = 1, itail = 0, iupdat = 0, iter = 0, nfgv = 0, ifun = 0, iback = 0;
  int nseg = 0, nintol = 0, nskip = 0, nfree = 0, nact = 0, ileave = 0, nenter = 0, iword = 0,
      info = 0;
  double theta = 1, fold = 0, tol = 0, dnorm = 0, epsmch = DBL_EPSILON, gd = 0, stpmx = 0,
         sbgnrm = 0, stp = 0, gdold = 0, dtd = 0, xstep = 0;
  // line search (dcsrch isave/dsave)
  bool ls_start = true, brackt = false;
  int stage = 1;
  double ginit = 0, gtest = 0, gx = 0, gy = 0, finit = 0, fx = 0, fy = 0, stx = 0, sty = 0,
         stmin = 0, stmax = 0, width = 0, width1 = 0;
  enum Csave { CS_START, CS_FG, CS_CONV, CS_WARN, CS_ERROR } csave = CS_START;
  // where to resume after the caller returns
  enum Resume { R_START, R_FG_START, R_FG_LN, R_NEW_X, R_DONE } resume = R_START;
  int last_task = 0;
  int last_nbreak = 0;  // breakpoints found by the last Cauchy search
  double f = 0.0;

  // 1-based accessors matching the Fortran
  double& WS(int i, int j) { return ws[(i - 1) + (size_t)n * (j - 1)]; }
  double& WY(int i, int j) { return wy[(i - 1) + (size_t)n * (j - 1)]; }
  double& SY(int i, int j) { return sy[(i - 1) + m * (j - 1)]; }
  double& SS(int i, int j) { return ss[(i - 1) + m * (j - 1)]; }
  double& WT(int i, int j) { return wt[(i - 1) + m * (j - 1)]; }
  double& WN(int i, int j) { return wn[(i - 1) + 2 * m * (j - 1)]; }
  double& WN1(int i, int j) { return snd[(i - 1) + 2 * m * (j - 1)]; }

  Lbfgsb(int n_, int m_, const double* l, const double* u, const int* nb, double fa, double pg)
      : n(n_), m(m_), lo(n_, 0.0), up(n_, 0.0), nbd(n_, 0), factr(fa), pgtol(pg) {
    for (int i = 0; i < n; ++i) {
      nbd[i] = nb ? nb[i] : 0;
      lo[i] = l ? l[i] : 0.0;
      up[i] = u ? u[i] : 0.0;
    }
    ws.assign((size_t)n * m, 0.0);
    wy.assign((size_t)n * m, 0.0);
    sy.assign(m * m, 0.0);
    ss.assign(m * m, 0.0);
    wt.assign(m * m, 0.0);
    wn.assign(4 * m * m, 0.0);
    snd.assign(4 * m * m, 0.0);
    z.assign(n, 0.0);
    r.assign(n, 0.0);
    d.assign(n, 0.0);
    t.assign(n, 0.0);
    xp.assign(n, 0.0);
    wa.assign(8 * m, 0.0);
    index.assign(n, 0);
    iwhere.assign(n, 0);
    indx2.assign(n, 0);
  }

  void reset_memory() {  // the "refresh the lbfgs memory" branches
    info = 0;
    col = 0;
    head = 1;
    theta = 1.0;
    iupdat = 0;
    updatd = false;
  }

  // ---- bmv (lbfgsb.f:1106-1220): product with the 2m x 2m middle matrix ----
  int bmv(const double* v, double* p) {
    if (col == 0) return 0;
    p[col] = v[col];
    for (int i = 2; i <= col; ++i) {
      double s = 0.0;
      for (int k = 1; k <= i - 1; ++k) s += SY(i, k) * v[k - 1] / SY(k, k);
      p[col + i - 1] = v[col + i - 1] + s;
    }
    if (tri_solve(wt.data(), m, col, p + col, true)) return -1;
    for (int i = 1; i <= col; ++i) p[i - 1] = v[i - 1] / std::sqrt(SY(i, i));
    if (tri_solve(wt.data(), m, col, p + col, false)) return -1;
    for (int i = 1; i <= col; ++i) p[i - 1] = -p[i - 1] / std::sqrt(SY(i, i));
    for (int i = 1; i <= col; ++i) {
      double s = 0.0;
      for (int k = i + 1; k <= col; ++k) s += SY(k, i) * p[col + k - 1] / SY(i, i);
      p[i - 1] += s;
    }
    return 0;
  }

  // ---- active (lbfgsb.f:1004-1104) ----
  void active(double* x) {
    prjctd = false;
    cnstnd = false;
    boxed = true;
    for (int i = 0; i < n; ++i) {
      if (nbd[i] > 0) {
        if (nbd[i] <= 2 && x[i] <= lo[i]) {
          if (x[i] < lo[i]) { prjctd = true; x[i] = lo[i]; }
        } else if (nbd[i] >= 2 && x[i] >= up[i]) {
          if (x[i] > up[i]) { prjctd = true; x[i] = up[i]; }
        }
      }
    }
    for (int i = 0; i < n; ++i) {
      if (nbd[i] != 2) boxed = false;
      if (nbd[i] == 0) {
        iwhere[i] = -1;
      } else {
        cnstnd = true;
        iwhere[i] = (nbd[i] == 2 && up[i] - lo[i] <= 0.0) ? 3 : 0;
      }
    }
  }

  // ---- projgr (lbfgsb.f:2942-2990) ----
  double projgr(const double* x, const double* g) {
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) {
      double gi = g[i];
      if (nbd[i] != 0) {
        if (gi < 0.0) {
          if (nbd[i] >= 2) gi = std::max(x[i] - up[i], gi);
        } else {
          if (nbd[i] <= 2) gi = std::min(x[i] - lo[i], gi);
        }
      }
      nrm = std::max(nrm, std::fabs(gi));
    }
    return nrm;
  }

  // ---- heap of breakpoints (hpsolb, lbfgsb.f:2341-2452) ----
  // tb[1..nh], ord[1..nh] (1-based views).  iheap==0 builds the heap first.
  static void heap_pop(int nh, double* tb, int* ord, int iheap) {
    if (iheap == 0) {
      for (int k = 2; k <= nh; ++k) {
        const double ddum = tb[k];
        const int in = ord[k];
        int i = k;
        while (i > 1) {
          const int j = i / 2;
          if (ddum < tb[j]) {
            tb[i] = tb[j];
            ord[i] = ord[j];
            i = j;
          } else {
            break;
          }
        }
        tb[i] = ddum;
        ord[i] = in;
      }
    }
    if (nh > 1) {
      int i = 1;
      const double out = tb[1];
      const int iout = ord[1];
      const double ddum = tb[nh];
      const int in = ord[nh];
      for (;;) {
        int j = i + i;
        if (j <= nh - 1) {
          if (tb[j + 1] < tb[j]) j = j + 1;
          if (tb[j] < ddum) {
            tb[i] = tb[j];
            ord[i] = ord[j];
            i = j;
            continue;
          }
        }
        break;
      }
      tb[i] = ddum;
      ord[i] = in;
      tb[nh] = out;
      ord[nh] = iout;
    }
  }

  // ---- cauchy (lbfgsb.f:1222-1719): generalized Cauchy point into z ----
  int cauchy(const double* x, const double* g) {
    double* p = wa.data();
    double* c = wa.data() + 2 * m;
    double* wbp = wa.data() + 4 * m;
    double* v = wa.data() + 6 * m;
    // iorder / t use 1-based views over indx2 / t
    int* iorder = indx2.data() - 1;
    double* tb = t.data() - 1;
    if (sbgnrm <= 0.0) {
      for (int i = 0; i < n; ++i) z[i] = x[i];
      return 0;
    }
    bool bnded = true;
    int nfr = n + 1, nbreak = 0, ibkmin = 0;
    double bkmin = 0.0, f1 = 0.0;
    const int col2 = 2 * col;
    for (int i = 0; i < col2; ++i) p[i] = 0.0;
    for (int i = 1; i <= n; ++i) {
      const double neggi = -g[i - 1];
      double tl = 0.0, tu = 0.0;
      if (iwhere[i - 1] != 3 && iwhere[i - 1] != -1) {
        if (nbd[i - 1] <= 2) tl = x[i - 1] - lo[i - 1];
        if (nbd[i - 1] >= 2) tu = up[i - 1] - x[i - 1];
        const bool xlower = nbd[i - 1] <= 2 && tl <= 0.0;
        const bool xupper = nbd[i - 1] >= 2 && tu <= 0.0;
        iwhere[i - 1] = 0;
        if (xlower) {
          if (neggi <= 0.0) iwhere[i - 1] = 1;
        } else if (xupper) {
          if (neggi >= 0.0) iwhere[i - 1] = 2;
        } else {
          if (std::fabs(neggi) <= 0.0) iwhere[i - 1] = -3;
        }
      }
      int pointr = head;
      if (iwhere[i - 1] != 0 && iwhere[i - 1] != -1) {
        d[i - 1] = 0.0;
      } else {
        d[i - 1] = neggi;
        f1 -= neggi * neggi;
        for (int j = 1; j <= col; ++j) {
          p[j - 1] += WY(i, pointr) * neggi;
          p[col + j - 1] += WS(i, pointr) * neggi;
          pointr = pointr % m + 1;
        }
        if (nbd[i - 1] <= 2 && nbd[i - 1] != 0 && neggi < 0.0) {
          ++nbreak;
          iorder[nbreak] = i;
          tb[nbreak] = tl / (-neggi);
          if (nbreak == 1 || tb[nbreak] < bkmin) {
            bkmin = tb[nbreak];
            ibkmin = nbreak;
          }
        } else if (nbd[i - 1] >= 2 && neggi > 0.0) {
          ++nbreak;
          iorder[nbreak] = i;
          tb[nbreak] = tu / neggi;
          if (nbreak == 1 || tb[nbreak] < bkmin) {
            bkmin = tb[nbreak];
            ibkmin = nbreak;
          }
        } else {
          --nfr;
          iorder[nfr] = i;
          if (std::fabs(neggi) > 0.0) bnded = false;
        }
      }
    }
    last_nbreak = nbreak;
    if (theta != 1.0)
      for (int j = 0; j < col; ++j) p[col + j] *= theta;
    for (int i = 0; i < n; ++i) z[i] = x[i];
    if (nbreak == 0 && nfr == n + 1) return 0;
    for (int j = 0; j < col2; ++j) c[j] = 0.0;
    double f2 = -theta * f1;
    const double f2_org = f2;
    if (col > 0) {
      if (bmv(p, v)) return -1;
      double s = 0.0;
      for (int j = 0; j < col2; ++j) s += v[j] * p[j];
      f2 -= s;
    }
    double dtm = -f1 / f2;
    double tsum = 0.0;
    nseg = 1;
    bool skip_to_999 = false;
    if (nbreak > 0) {
      int nleft = nbreak, it = 1;
      double tj = 0.0;
      for (;;) {
        const double tj0 = tj;
        int ibp;
        if (it == 1) {
          tj = bkmin;
          ibp = iorder[ibkmin];
        } else {
          if (it == 2 && ibkmin != nbreak) {
            tb[ibkmin] = tb[nbreak];
            iorder[ibkmin] = iorder[nbreak];
          }
          heap_pop(nleft, tb, iorder, it - 2);
          tj = tb[nleft];
          ibp = iorder[nleft];
        }
        const double dt = tj - tj0;
        if (dtm < dt) break;
        tsum += dt;
        --nleft;
        ++it;
        const double dibp = d[ibp - 1];
        d[ibp - 1] = 0.0;
        double zibp;
        if (dibp > 0.0) {
          zibp = up[ibp - 1] - x[ibp - 1];
          z[ibp - 1] = up[ibp - 1];
          iwhere[ibp - 1] = 2;
        } else {
          zibp = lo[ibp - 1] - x[ibp - 1];
          z[ibp - 1] = lo[ibp - 1];
          iwhere[ibp - 1] = 1;
        }
        if (nleft == 0 && nbreak == n) {
          dtm = dt;
          skip_to_999 = true;
          break;
        }
        ++nseg;
        const double dibp2 = dibp * dibp;
        f1 = f1 + dt * f2 + dibp2 - theta * dibp * zibp;
        f2 = f2 - theta * dibp2;
        if (col > 0) {
          for (int j = 0; j < col2; ++j) c[j] += dt * p[j];
          int pointr = head;
          for (int j = 1; j <= col; ++j) {
            wbp[j - 1] = WY(ibp, pointr);
            wbp[col + j - 1] = theta * WS(ibp, pointr);
            pointr = pointr % m + 1;
          }
          if (bmv(wbp, v)) return -1;
          double wmc = 0, wmp = 0, wmw = 0;
          for (int j = 0; j < col2; ++j) {
            wmc += c[j] * v[j];
            wmp += p[j] * v[j];
            wmw += wbp[j] * v[j];
          }
          for (int j = 0; j < col2; ++j) p[j] -= dibp * wbp[j];
          f1 += dibp * wmc;
          f2 += 2.0 * dibp * wmp - dibp2 * wmw;
        }
        f2 = std::max(epsmch * f2_org, f2);
        if (nleft > 0) {
          dtm = -f1 / f2;
          continue;
        } else if (bnded) {
          f1 = 0.0;
          f2 = 0.0;
          dtm = 0.0;
        } else {
          dtm = -f1 / f2;
        }
        break;
      }
    }
    if (!skip_to_999) {
      if (dtm <= 0.0) dtm = 0.0;
      tsum += dtm;
      for (int i = 0; i < n; ++i) z[i] += tsum * d[i];
    }
    if (col > 0)
      for (int j = 0; j < col2; ++j) c[j] += dtm * p[j];
    return 0;
  }

  // ---- freev (lbfgsb.f:2241-2340) ----
  void freev() {
    nenter = 0;
    ileave = n + 1;
    if (iter > 0 && cnstnd) {
      for (int i = 1; i <= nfree; ++i) {
        const int k = index[i - 1];
        if (iwhere[k - 1] > 0) {
          --ileave;
          indx2[ileave - 1] = k;
        }
      }
      for (int i = 1 + nfree; i <= n; ++i) {
        const int k = index[i - 1];
        if (iwhere[k - 1] <= 0) {
          ++nenter;
          indx2[nenter - 1] = k;
        }
      }
    }
    wrk = (ileave < n + 1) || (nenter > 0) || updatd;
    nfree = 0;
    int iact = n + 1;
    for (int i = 1; i <= n; ++i) {
      if (iwhere[i - 1] <= 0) {
        ++nfree;
        index[nfree - 1] = i;
      } else {
        --iact;
        index[iact - 1] = i;
      }
    }
  }

  // ---- formk (lbfgsb.f:1848-2172) ----
  int formk() {
    const int nsub = nfree;
    if (updatd) {
      if (iupdat > m) {
        for (int jy = 1; jy <= m - 1; ++jy) {
          const int js = m + jy;
          for (int k = 0; k < m - jy; ++k) WN1(jy + k, jy) = WN1(jy + 1 + k, jy + 1);
          for (int k = 0; k < m - jy; ++k) WN1(js + k, js) = WN1(js + 1 + k, js + 1);
          for (int k = 0; k < m - 1; ++k) WN1(m + 1 + k, jy) = WN1(m + 2 + k, jy + 1);
        }
      }
      const int pbegin = 1, pend = nsub, dbegin = nsub + 1, dend = n;
      int iy = col, is = m + col;
      int ipntr = head + col - 1;
      if (ipntr > m) ipntr -= m;
      int jpntr = head;
      for (int jy = 1; jy <= col; ++jy) {
        const int js = m + jy;
        double t1 = 0, t2 = 0, t3 = 0;
        for (int k = pbegin; k <= pend; ++k) {
          const int k1 = index[k - 1];
          t1 += WY(k1, ipntr) * WY(k1, jpntr);
        }
        for (int k = dbegin; k <= dend; ++k) {
          const int k1 = index[k - 1];
          t2 += WS(k1, ipntr) * WS(k1, jpntr);
          t3 += WS(k1, ipntr) * WY(k1, jpntr);
        }
        WN1(iy, jy) = t1;
        WN1(is, js) = t2;
        WN1(is, jy) = t3;
        jpntr = jpntr % m + 1;
      }
      const int jy = col;
      jpntr = head + col - 1;
      if (jpntr > m) jpntr -= m;
      ipntr = head;
      for (int i = 1; i <= col; ++i) {
        const int is2 = m + i;
        double t3 = 0;
        for (int k = pbegin; k <= pend; ++k) {
          const int k1 = index[k - 1];
          t3 += WS(k1, ipntr) * WY(k1, jpntr);
        }
        ipntr = ipntr % m + 1;
        WN1(is2, jy) = t3;
      }
    }
    const int upcl = updatd ? col - 1 : col;
    int ipntr = head;
    for (int iy = 1; iy <= upcl; ++iy) {
      const int is = m + iy;
      int jpntr = head;
      for (int jy = 1; jy <= iy; ++jy) {
        const int js = m + jy;
        double t1 = 0, t2 = 0, t3 = 0, t4 = 0;
        for (int k = 1; k <= nenter; ++k) {
          const int k1 = indx2[k - 1];
          t1 += WY(k1, ipntr) * WY(k1, jpntr);
          t2 += WS(k1, ipntr) * WS(k1, jpntr);
        }
        for (int k = ileave; k <= n; ++k) {
          const int k1 = indx2[k - 1];
          t3 += WY(k1, ipntr) * WY(k1, jpntr);
          t4 += WS(k1, ipntr) * WS(k1, jpntr);
        }
        WN1(iy, jy) = WN1(iy, jy) + t1 - t3;
        WN1(is, js) = WN1(is, js) - t2 + t4;
        jpntr = jpntr % m + 1;
      }
      ipntr = ipntr % m + 1;
    }
    ipntr = head;
    for (int is = m + 1; is <= m + upcl; ++is) {
      int jpntr = head;
      for (int jy = 1; jy <= upcl; ++jy) {
        double t1 = 0, t3 = 0;
        for (int k = 1; k <= nenter; ++k) {
          const int k1 = indx2[k - 1];
          t1 += WS(k1, ipntr) * WY(k1, jpntr);
        }
        for (int k = ileave; k <= n; ++k) {
          const int k1 = indx2[k - 1];
          t3 += WS(k1, ipntr) * WY(k1, jpntr);
        }
        if (is <= jy + m)
          WN1(is, jy) = WN1(is, jy) + t1 - t3;
        else
          WN1(is, jy) = WN1(is, jy) - t1 + t3;
        jpntr = jpntr % m + 1;
      }
      ipntr = ipntr % m + 1;
    }
    const int m2 = 2 * m;
    for (int iy = 1; iy <= col; ++iy) {
      const int is = col + iy, is1 = m + iy;
      for (int jy = 1; jy <= iy; ++jy) {
        const int js = col + jy, js1 = m + jy;
        WN(jy, iy) = WN1(iy, jy) / theta;
        WN(js, is) = WN1(is1, js1) * theta;
      }
      for (int jy = 1; jy <= iy - 1; ++jy) WN(jy, is) = -WN1(is1, jy);
      for (int jy = iy; jy <= col; ++jy) WN(jy, is) = WN1(is1, jy);
      WN(iy, iy) = WN(iy, iy) + SY(iy, iy);
    }
    if (chol_upper(wn.data(), m2, col)) return -1;
    const int col2 = 2 * col;
    for (int js = col + 1; js <= col2; ++js) tri_solve(wn.data(), m2, col, &WN(1, js), true);
    for (int is = col + 1; is <= col2; ++is)
      for (int js = is; js <= col2; ++js) {
        double s = 0;
        for (int k = 1; k <= col; ++k) s += WN(k, is) * WN(k, js);
        WN(is, js) = WN(is, js) + s;
      }
    if (chol_upper(&WN(col + 1, col + 1), m2, col)) return -2;
    return 0;
  }

  // ---- cmprlb (lbfgsb.f:1720-1786) ----
  int cmprlb(const double* x, const double* g) {
    if (!cnstnd && col > 0) {
      for (int i = 0; i < n; ++i) r[i] = -g[i];
      return 0;
    }
    for (int i = 1; i <= nfree; ++i) {
      const int k = index[i - 1];
      r[i - 1] = -theta * (z[k - 1] - x[k - 1]) - g[k - 1];
    }
    if (bmv(wa.data() + 2 * m, wa.data())) return -8;
    int pointr = head;
    for (int j = 1; j <= col; ++j) {
      const double a1 = wa[j - 1], a2 = theta * wa[col + j - 1];
      for (int i = 1; i <= nfree; ++i) {
        const int k = index[i - 1];
        r[i - 1] += WY(k, pointr) * a1 + WS(k, pointr) * a2;
      }
      pointr = pointr % m + 1;
    }
    return 0;
  }

  // ---- subsm (lbfgsb.f:2991-3346) with the 2011 projection ----
  int subsm(const double* xx, const double* gg) {
    // "d" of subsm is r (indexed by free position), "x" is the Cauchy point z
    const int nsub = nfree;
    if (nsub <= 0) return 0;
    double* wv = wa.data();
    int pointr = head;
    for (int i = 1; i <= col; ++i) {
      double t1 = 0, t2 = 0;
      for (int j = 1; j <= nsub; ++j) {
        const int k = index[j - 1];
        t1 += WY(k, pointr) * r[j - 1];
        t2 += WS(k, pointr) * r[j - 1];
      }
      wv[i - 1] = t1;
      wv[col + i - 1] = theta * t2;
      pointr = pointr % m + 1;
    }
    const int m2 = 2 * m, col2 = 2 * col;
    if (tri_solve(wn.data(), m2, col2, wv, true)) return -1;
    for (int i = 0; i < col; ++i) wv[i] = -wv[i];
    if (tri_solve(wn.data(), m2, col2, wv, false)) return -1;
    pointr = head;
    for (int jy = 1; jy <= col; ++jy) {
      const int js = col + jy;
      for (int i = 1; i <= nsub; ++i) {
        const int k = index[i - 1];
        r[i - 1] += WY(k, pointr) * wv[jy - 1] / theta + WS(k, pointr) * wv[js - 1];
      }
      pointr = pointr % m + 1;
    }
    for (int i = 0; i < nsub; ++i) r[i] *= 1.0 / theta;
    iword = 0;
    for (int i = 0; i < n; ++i) xp[i] = z[i];
    for (int i = 1; i <= nsub; ++i) {
      const int k = index[i - 1];
      const double dk = r[i - 1];
      double xk = z[k - 1];
      const int nb = nbd[k - 1];
      if (nb != 0) {
        if (nb == 1) {
          z[k - 1] = std::max(lo[k - 1], xk + dk);
          if (z[k - 1] == lo[k - 1]) iword = 1;
        } else if (nb == 2) {
          xk = std::max(lo[k - 1], xk + dk);
          z[k - 1] = std::min(up[k - 1], xk);
          if (z[k - 1] == lo[k - 1] || z[k - 1] == up[k - 1]) iword = 1;
        } else if (nb == 3) {
          z[k - 1] = std::min(up[k - 1], xk + dk);
          if (z[k - 1] == up[k - 1]) iword = 1;
        }
      } else {
        z[k - 1] = xk + dk;
      }
    }
    if (iword == 0) return 0;
    double dd_p = 0.0;
    for (int i = 0; i < n; ++i) dd_p += (z[i] - xx[i]) * gg[i];
    if (dd_p <= 0.0) return 0;
    for (int i = 0; i < n; ++i) z[i] = xp[i];
    double alpha = 1.0, temp1 = alpha;
    int ibd = 0;
    for (int i = 1; i <= nsub; ++i) {
      const int k = index[i - 1];
      const double dk = r[i - 1];
      const int nb = nbd[k - 1];
      if (nb != 0) {
        if (dk < 0.0 && nb <= 2) {
          const double temp2 = lo[k - 1] - z[k - 1];
          if (temp2 >= 0.0)
            temp1 = 0.0;
          else if (dk * alpha < temp2)
            temp1 = temp2 / dk;
        } else if (dk > 0.0 && nb >= 2) {
          const double temp2 = up[k - 1] - z[k - 1];
          if (temp2 <= 0.0)
            temp1 = 0.0;
          else if (dk * alpha > temp2)
            temp1 = temp2 / dk;
        }
        if (temp1 < alpha) {
          alpha = temp1;
          ibd = i;
        }
      }
    }
    if (alpha < 1.0) {
      const double dk = r[ibd - 1];
      const int k = index[ibd - 1];
      if (dk > 0.0) {
        z[k - 1] = up[k - 1];
        r[ibd - 1] = 0.0;
      } else if (dk < 0.0) {
        z[k - 1] = lo[k - 1];
        r[ibd - 1] = 0.0;
      }
    }
    for (int i = 1; i <= nsub; ++i) {
      const int k = index[i - 1];
      z[k - 1] += alpha * r[i - 1];
    }
    return 0;
  }

  // ---- matupd (lbfgsb.f:2584-2670) ----
  void matupd(double rr, double dr) {
    if (iupdat <= m) {
      col = iupdat;
      itail = (head + iupdat - 2) % m + 1;
    } else {
      itail = itail % m + 1;
      head = head % m + 1;
    }
    for (int i = 1; i <= n; ++i) {
      WS(i, itail) = d[i - 1];
      WY(i, itail) = r[i - 1];
    }
    theta = rr / dr;
    if (iupdat > m) {
      for (int j = 1; j <= col - 1; ++j) {
        for (int k = 0; k < j; ++k) SS(1 + k, j) = SS(2 + k, j + 1);
        for (int k = 0; k < col - j; ++k) SY(j + k, j) = SY(j + 1 + k, j + 1);
      }
    }
    int pointr = head;
    for (int j = 1; j <= col - 1; ++j) {
      double a = 0, b = 0;
      for (int i = 1; i <= n; ++i) {
        a += d[i - 1] * WY(i, pointr);
        b += WS(i, pointr) * d[i - 1];
      }
      SY(col, j) = a;
      SS(j, col) = b;
      pointr = pointr % m + 1;
    }
    SS(col, col) = (stp == 1.0) ? dtd : stp * stp * dtd;
    SY(col, col) = dr;
  }

  // ---- formt (lbfgsb.f:2173-2240) ----
  int formt() {
    for (int j = 1; j <= col; ++j) WT(1, j) = theta * SS(1, j);
    for (int i = 2; i <= col; ++i)
      for (int j = i; j <= col; ++j) {
        const int k1 = std::min(i, j) - 1;
        double dd = 0.0;
        for (int k = 1; k <= k1; ++k) dd += SY(i, k) * SY(j, k) / SY(k, k);
        WT(i, j) = dd + theta * SS(i, j);
      }
    return chol_upper(wt.data(), m, col) ? -3 : 0;
  }

  // ---- dcstep (lbfgsb.f:3694-3949) ----
  static void dcstep(double& stx_, double& fx_, double& dx, double& sty_, double& fy_, double& dy,
                     double& stp_, double fp, double dp, bool& brackt_, double stpmin,
                     double stpmax) {
    const double sgnd = dp * (dx / std::fabs(dx));
    double stpf, stpc, stpq;
    if (fp > fx_) {
      const double th = 3.0 * (fx_ - fp) / (stp_ - stx_) + dx + dp;
      const double s = std::max(std::fabs(th), std::max(std::fabs(dx), std::fabs(dp)));
      double gam = s * std::sqrt((th / s) * (th / s) - (dx / s) * (dp / s));
      if (stp_ < stx_) gam = -gam;
      const double p = (gam - dx) + th;
      const double q = ((gam - dx) + gam) + dp;
      const double rr = p / q;
      stpc = stx_ + rr * (stp_ - stx_);
      stpq = stx_ + ((dx / ((fx_ - fp) / (stp_ - stx_) + dx)) / 2.0) * (stp_ - stx_);
      if (std::fabs(stpc - stx_) < std::fabs(stpq - stx_))
        stpf = stpc;
      else
        stpf = stpc + (stpq - stpc) / 2.0;
      brackt_ = true;
    } else if (sgnd < 0.0) {
      const double th = 3.0 * (fx_ - fp) / (stp_ - stx_) + dx + dp;
      const double s = std::max(std::fabs(th), std::max(std::fabs(dx), std::fabs(dp)));
      double gam = s * std::sqrt((th / s) * (th / s) - (dx / s) * (dp / s));
      if (stp_ > stx_) gam = -gam;
      const double p = (gam - dp) + th;
      const double q = ((gam - dp) + gam) + dx;
      const double rr = p / q;
      stpc = stp_ + rr * (stx_ - stp_);
      stpq = stp_ + (dp / (dp - dx)) * (stx_ - stp_);
      stpf = (std::fabs(stpc - stp_) > std::fabs(stpq - stp_)) ? stpc : stpq;
      brackt_ = true;
    } else if (std::fabs(dp) < std::fabs(dx)) {
      const double th = 3.0 * (fx_ - fp) / (stp_ - stx_) + dx + dp;
      const double s = std::max(std::fabs(th), std::max(std::fabs(dx), std::fabs(dp)));
      double gam = s * std::sqrt(std::max(0.0, (th / s) * (th / s) - (dx / s) * (dp / s)));
      if (stp_ > stx_) gam = -gam;
      const double p = (gam - dp) + th;
      const double q = (gam + (dx - dp)) + gam;
      const double rr = p / q;
      if (rr < 0.0 && gam != 0.0)
        stpc = stp_ + rr * (stx_ - stp_);
      else if (stp_ > stx_)
        stpc = stpmax;
      else
        stpc = stpmin;
      stpq = stp_ + (dp / (dp - dx)) * (stx_ - stp_);
      if (brackt_) {
        stpf = (std::fabs(stpc - stp_) < std::fabs(stpq - stp_)) ? stpc : stpq;
        if (stp_ > stx_)
          stpf = std::min(stp_ + 0.66 * (sty_ - stp_), stpf);
        else
          stpf = std::max(stp_ + 0.66 * (sty_ - stp_), stpf);
      } else {
        stpf = (std::fabs(stpc - stp_) > std::fabs(stpq - stp_)) ? stpc : stpq;
        stpf = std::min(stpmax, stpf);
        stpf = std::max(stpmin, stpf);
      }
    } else {
      if (brackt_) {
        const double th = 3.0 * (fp - fy_) / (sty_ - stp_) + dy + dp;
        const double s = std::max(std::fabs(th), std::max(std::fabs(dy), std::fabs(dp)));
        double gam = s * std::sqrt((th / s) * (th / s) - (dy / s) * (dp / s));
        if (stp_ > sty_) gam = -gam;
        const double p = (gam - dp) + th;
        const double q = ((gam - dp) + gam) + dy;
        const double rr = p / q;
        stpc = stp_ + rr * (sty_ - stp_);
        stpf = stpc;
      } else if (stp_ > stx_) {
        stpf = stpmax;
      } else {
        stpf = stpmin;
      }
    }
    if (fp > fx_) {
      sty_ = stp_;
      fy_ = fp;
      dy = dp;
    } else {
      if (sgnd < 0.0) {
        sty_ = stx_;
        fy_ = fx_;
        dy = dx;
      }
      stx_ = stp_;
      fx_ = fp;
      dx = dp;
    }
    stp_ = stpf;
  }

  // ---- dcsrch (lbfgsb.f:3347-3693), ftol=1e-3 gtol=0.9 xtol=0.1 ----
  void dcsrch(double fv, double gv, double stpmin, double stpmax) {
    const double ftol = 1e-3, gtl = 0.9, xtol = 0.1;
    if (csave == CS_START) {
      if (stp < stpmin || stp > stpmax || gv >= 0.0 || stpmax < stpmin) {
        csave = CS_ERROR;
        return;
      }
      brackt = false;
      stage = 1;
      finit = fv;
      ginit = gv;
      gtest = ftol * ginit;
      width = stpmax - stpmin;
      width1 = width / 0.5;
      stx = 0.0;
      fx = finit;
      gx = ginit;
      sty = 0.0;
      fy = finit;
      gy = ginit;
      stmin = 0.0;
      stmax = stp + 4.0 * stp;
      csave = CS_FG;
      return;
    }
    const double ftest = finit + stp * gtest;
    if (stage == 1 && fv <= ftest && gv >= 0.0) stage = 2;
    Csave task = CS_FG;
    if (brackt && (stp <= stmin || stp >= stmax)) task = CS_WARN;
    if (brackt && stmax - stmin <= xtol * stmax) task = CS_WARN;
    if (stp == stpmax && fv <= ftest && gv <= gtest) task = CS_WARN;
    if (stp == stpmin && (fv > ftest || gv >= gtest)) task = CS_WARN;
    if (fv <= ftest && std::fabs(gv) <= gtl * (-ginit)) task = CS_CONV;
    if (task == CS_WARN || task == CS_CONV) {
      csave = task;
      return;
    }
    if (stage == 1 && fv <= fx && fv > ftest) {
      double fm = fv - stp * gtest;
      double fxm = fx - stx * gtest;
      double fym = fy - sty * gtest;
      double gm = gv - gtest;
      double gxm = gx - gtest;
      double gym = gy - gtest;
      dcstep(stx, fxm, gxm, sty, fym, gym, stp, fm, gm, brackt, stmin, stmax);
      fx = fxm + stx * gtest;
      fy = fym + sty * gtest;
      gx = gxm + gtest;
      gy = gym + gtest;
    } else {
      dcstep(stx, fx, gx, sty, fy, gy, stp, fv, gv, brackt, stmin, stmax);
    }
    if (brackt) {
      if (std::fabs(sty - stx) >= 0.66 * width1) stp = stx + 0.5 * (sty - stx);
      width1 = width;
      width = std::fabs(sty - stx);
    }
    if (brackt) {
      stmin = std::min(stx, sty);
      stmax = std::max(stx, sty);
    } else {
      stmin = stp + 1.1 * (stp - stx);
      stmax = stp + 4.0 * (stp - stx);
    }
    stp = std::max(stp, stpmin);
    stp = std::min(stp, stpmax);
    if ((brackt && (stp <= stmin || stp >= stmax)) || (brackt && stmax - stmin <= xtol * stmax))
      stp = stx;
    csave = CS_FG;
  }

  // lnsrlb first part (lbfgsb.f:2453-2535): returns false on info != 0
  void lnsrlb_init(const double* x, const double* g) {
    dtd = 0.0;
    for (int i = 0; i < n; ++i) dtd += d[i] * d[i];
    dnorm = std::sqrt(dtd);
    stpmx = kBig;
    if (cnstnd) {
      if (iter == 0) {
        stpmx = 1.0;
      } else {
        for (int i = 0; i < n; ++i) {
          const double a1 = d[i];
          if (nbd[i] != 0) {
            if (a1 < 0.0 && nbd[i] <= 2) {
              const double a2 = lo[i] - x[i];
              if (a2 >= 0.0)
                stpmx = 0.0;
              else if (a1 * stpmx < a2)
                stpmx = a2 / a1;
            } else if (a1 > 0.0 && nbd[i] >= 2) {
              const double a2 = up[i] - x[i];
              if (a2 <= 0.0)
                stpmx = 0.0;
              else if (a1 * stpmx > a2)
                stpmx = a2 / a1;
            }
          }
        }
      }
    }
    stp = (iter == 0 && !boxed) ? std::min(1.0 / dnorm, stpmx) : 1.0;
    for (int i = 0; i < n; ++i) {
      t[i] = x[i];
      r[i] = g[i];
    }
    fold = f;
    ifun = 0;
    iback = 0;
    csave = CS_START;
  }

  // lnsrlb from label 556: returns 1 if an evaluation is requested, 0 if the
  // search finished (NEW_X), -1 on failure (info set).
  int lnsrlb_continue(double* x, const double* g) {
    gd = 0.0;
    for (int i = 0; i < n; ++i) gd += g[i] * d[i];
    if (ifun == 0) {
      gdold = gd;
      if (gd >= 0.0) {
        info = -4;
        return -1;
      }
    }
    dcsrch(f, gd, 0.0, stpmx);
    if (csave == CS_ERROR) {
      // dcsrch's ERROR task is neither CONV nor WARN: lnsrlb keeps asking for
      // evaluations at the unchanged stp (lbfgsb.f:2560-2575)
    }
    xstep = stp * dnorm;
    if (csave != CS_CONV && csave != CS_WARN) {
      ++ifun;
      ++nfgv;
      iback = ifun - 1;
      if (stp == 1.0) {
        for (int i = 0; i < n; ++i) x[i] = z[i];
      } else {
        for (int i = 0; i < n; ++i) x[i] = stp * d[i] + t[i];
      }
      return 1;
    }
    return 0;
  }

  // The body of mainlb from label 222 to the line search request.
  // Returns the task to hand back to the caller.
  int iterate_from_222(double* x, const double* g) {
    for (;;) {  // label 222
      iword = -1;
      bool goto333 = false;
      if (!cnstnd && col > 0) {
        for (int i = 0; i < n; ++i) z[i] = x[i];
        wrk = updatd;
        nseg = 0;
        goto333 = true;
      }
      if (!goto333) {
        if (cauchy(x, g) != 0) {
          reset_memory();
          continue;
        }
        nintol += nseg;
        freev();
        nact = n - nfree;
      }
      // label 333
      if (!(nfree == 0 || col == 0)) {
        if (wrk && formk() != 0) {
          reset_memory();
          continue;
        }
        int rc = cmprlb(x, g);
        if (rc == 0) rc = subsm(x, g);
        if (rc != 0) {
          reset_memory();
          continue;
        }
      }
      // label 555
      for (int i = 0; i < n; ++i) d[i] = z[i] - x[i];
      lnsrlb_init(x, g);
      const int rc = lnsrlb_continue(x, g);
      if (rc < 0) {
        int res = line_search_failed(x, const_cast<double*>(g));
        if (res == 1) continue;  // restart at 222
        return res;
      }
      if (rc == 1) {
        resume = R_FG_LN;
        return ORC_TASK_FG;
      }
      // line search converged without an evaluation (not reachable on the
      // first call since csave START always asks for one); treat as NEW_X
      return finish_iteration(x, g);
    }
  }

  // mainlb's "info /= 0 or iback >= 20" branch.  Returns 1 to restart at 222
  // or a terminal task.
  int line_search_failed(double* x, double* g) {
    for (int i = 0; i < n; ++i) {
      x[i] = t[i];
      g[i] = r[i];
    }
    f = fold;
    if (col == 0) {
      if (info == 0) {
        info = -9;
        --nfgv;
        --ifun;
        --iback;
      }
      ++iter;
      resume = R_DONE;
      return ORC_TASK_ABNORMAL;
    }
    if (info == 0) --nfgv;
    reset_memory();
    return 1;
  }

  int finish_iteration(const double* x, const double* g) {
    ++iter;
    sbgnrm = projgr(x, g);
    resume = R_NEW_X;
    return ORC_TASK_NEW_X;
  }

  // setulb entry point
  int step(double* x, double fval, double* g) {
    f = fval;
    switch (resume) {
      case R_START: {
        tol = factr * epsmch;
        if (n <= 0 || m <= 0 || factr < 0.0) {
          resume = R_DONE;
          return last_task = ORC_TASK_ERROR;
        }
        for (int i = 0; i < n; ++i) {
          if (nbd[i] < 0 || nbd[i] > 3 || (nbd[i] == 2 && lo[i] > up[i])) {
            resume = R_DONE;
            return last_task = ORC_TASK_ERROR;
          }
        }
        active(x);
        nfree = n;
        resume = R_FG_START;
        return last_task = ORC_TASK_FG;
      }
      case R_FG_START: {
        nfgv = 1;
        sbgnrm = projgr(x, g);
        if (sbgnrm <= pgtol) {
          resume = R_DONE;
          return last_task = ORC_TASK_CONV;
        }
        return last_task = iterate_from_222(x, g);
      }
      case R_FG_LN: {
        const int rc = lnsrlb_continue(x, g);
        if (rc < 0 || iback >= 20) {
          const int res = line_search_failed(x, g);
          if (res == 1) return last_task = iterate_from_222(x, g);
          return last_task = res;
        }
        if (rc == 1) return last_task = ORC_TASK_FG;
        return last_task = finish_iteration(x, g);
      }
      case R_NEW_X: {
        if (sbgnrm <= pgtol) {
          resume = R_DONE;
          return last_task = ORC_TASK_CONV;
        }
        const double ddum = std::max(std::fabs(fold), std::max(std::fabs(f), 1.0));
        if ((fold - f) <= tol * ddum) {
          resume = R_DONE;
          return last_task = ORC_TASK_CONV;
        }
        for (int i = 0; i < n; ++i) r[i] = g[i] - r[i];
        double rr = 0.0;
        for (int i = 0; i < n; ++i) rr += r[i] * r[i];
        double dr, dd;
        if (stp == 1.0) {
          dr = gd - gdold;
          dd = -gdold;
        } else {
          dr = (gd - gdold) * stp;
          for (int i = 0; i < n; ++i) d[i] *= stp;
          dd = -gdold * stp;
        }
        if (dr <= epsmch * dd) {
          ++nskip;
          updatd = false;
        } else {
          updatd = true;
          ++iupdat;
          matupd(rr, dr);
          if (formt() != 0) reset_memory();
        }
        return last_task = iterate_from_222(x, g);
      }
      case R_DONE:
      default:
        return last_task;
    }
  }
};

}  // namespace

extern "C" void* orc_lbfgsb_new(int n, int m, const double* l, const double* u, const int* nbd,
                                double factr, double pgtol) {
  return new Lbfgsb(n, m, l, u, nbd, factr, pgtol);
}

extern "C" int orc_lbfgsb_step(void* h, double* x, double f, const double* g) {
  Lbfgsb* s = static_cast<Lbfgsb*>(h);
  // the solver may restore g on a failed line search, so work on a copy
  static thread_local std::vector<double> gbuf;
  gbuf.assign(g, g + s->n);
  return s->step(x, f, gbuf.data());
}

extern "C" int orc_lbfgsb_info(void* h, int* iter, int* nfgv, int* col, double* theta,
                               double* sbgnrm) {
  Lbfgsb* s = static_cast<Lbfgsb*>(h);
  if (iter && nfgv && col == nullptr && theta == nullptr && sbgnrm == nullptr) {
    // diagnostic form: report (nseg, nbreak) of the last Cauchy search
    *iter = s->nseg;
    *nfgv = s->last_nbreak;
    return 1;
  }
  if (iter) *iter = s->iter;
  if (nfgv) *nfgv = s->nfgv;
  if (col) *col = s->col;
  if (theta) *theta = s->theta;
  if (sbgnrm) *sbgnrm = s->sbgnrm;
  return 0;
}

extern "C" void orc_lbfgsb_free(void* h) { delete static_cast<Lbfgsb*>(h); }
