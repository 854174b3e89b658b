/*
 * Test infrastructure only (CPU oracle / CPU baseline build of the G2S
 * reference): project-written implementation of the FFTW3 single-precision
 * API subset declared in fftw3.h.  It is NOT FFTW: it is a self-sorting
 * (Stockham) mixed-radix FFT written for this repository, so that the
 * reference's own CPU QuickSampling sources can be compiled and run in an
 * image where libfftw3f is absent.  Transforms are unnormalised and use the
 * FFTW array conventions (row-major, last dimension halved for r2c/c2r).
 *
 * Algorithm: decimation-in-frequency Stockham autosort.  A length-n stage of
 * radix p with stride s maps x -> y by
 *     a_r = x[q + s*(t + r*m)],   m = n/p,
 *     y[q + s*(p*t + k)] = (DFT_p a)_k * exp(sign*2*pi*i*t*k/n),
 * then recurses on length m with stride s*p.  Real transforms of even length
 * use the half-length complex transform plus the standard split twiddles.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define restrict __restrict__

typedef struct { float r, i; } cpx;

/* ------------------------------------------------------------------ */
/* 1-D complex plan                                                    */
/* ------------------------------------------------------------------ */
#define MAX_STAGES 40

typedef struct {
    int n;
    int sign;
    int nstage;
    int radix[MAX_STAGES];
    cpx *tw[MAX_STAGES];     /* per stage: m*(p-1) twiddles */
    cpx *wp[MAX_STAGES];     /* per stage: p*p DFT matrix for generic radices */
    cpx *bufa, *bufb;        /* work buffers (length n) */
} cplan;

static void cplan_init(cplan *pl, int n, int sign) {
    memset(pl, 0, sizeof(*pl));
    pl->n = n;
    pl->sign = sign;
    int rem = n;
    while (rem > 1) {
        int p;
        if (rem % 4 == 0) p = 4;
        else if (rem % 2 == 0) p = 2;
        else if (rem % 3 == 0) p = 3;
        else if (rem % 5 == 0) p = 5;
        else if (rem % 7 == 0) p = 7;
        else {
            p = rem;
            for (int d = 11; (long)d * d <= rem; d += 2)
                if (rem % d == 0) { p = d; break; }
        }
        pl->radix[pl->nstage++] = p;
        rem /= p;
    }
    int len = n;
    for (int st = 0; st < pl->nstage; ++st) {
        int p = pl->radix[st];
        int m = len / p;
        pl->tw[st] = (cpx *)malloc(sizeof(cpx) * (size_t)(m * (p - 1) + 1));
        for (int t = 0; t < m; ++t)
            for (int k = 1; k < p; ++k) {
                double ang = sign * 2.0 * M_PI * (double)t * (double)k / (double)len;
                pl->tw[st][t * (p - 1) + (k - 1)].r = (float)cos(ang);
                pl->tw[st][t * (p - 1) + (k - 1)].i = (float)sin(ang);
            }
        if (p != 2 && p != 4 && p != 3) {
            pl->wp[st] = (cpx *)malloc(sizeof(cpx) * (size_t)(p * p));
            for (int k = 0; k < p; ++k)
                for (int r = 0; r < p; ++r) {
                    double ang = sign * 2.0 * M_PI * (double)((k * r) % p) / (double)p;
                    pl->wp[st][k * p + r].r = (float)cos(ang);
                    pl->wp[st][k * p + r].i = (float)sin(ang);
                }
        }
        len = m;
    }
    pl->bufa = (cpx *)malloc(sizeof(cpx) * (size_t)(n > 0 ? n : 1));
    pl->bufb = (cpx *)malloc(sizeof(cpx) * (size_t)(n > 0 ? n : 1));
}

static void cplan_free(cplan *pl) {
    for (int st = 0; st < pl->nstage; ++st) {
        free(pl->tw[st]);
        free(pl->wp[st]);
    }
    free(pl->bufa);
    free(pl->bufb);
}

static inline cpx cmul(cpx a, cpx b) {
    cpx c = {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r};
    return c;
}

/* One Stockham stage on a batch: element j of vector b lives at x[j*B + b].
 * x (length n, stride s) -> y.  The innermost loop runs over the batch so
 * that it vectorises. */
static void stage(const cplan *pl, int st, int n, int s, int B, const cpx *restrict x, cpx *restrict y) {
    const int p = pl->radix[st];
    const int m = n / p;
    const cpx *tw = pl->tw[st];
    const float sg = (float)pl->sign;
    if (p == 2) {
        for (int t = 0; t < m; ++t) {
            const cpx w1 = tw[t];
            for (int q = 0; q < s; ++q) {
                const cpx *a0p = x + (size_t)(q + s * t) * B, *a1p = x + (size_t)(q + s * (t + m)) * B;
                cpx *y0 = y + (size_t)(q + s * (2 * t)) * B, *y1 = y + (size_t)(q + s * (2 * t + 1)) * B;
                for (int b = 0; b < B; ++b) {
                    cpx a0 = a0p[b], a1 = a1p[b];
                    float dr = a0.r - a1.r, di = a0.i - a1.i;
                    y0[b].r = a0.r + a1.r; y0[b].i = a0.i + a1.i;
                    y1[b].r = dr * w1.r - di * w1.i; y1[b].i = dr * w1.i + di * w1.r;
                }
            }
        }
    } else if (p == 4) {
        for (int t = 0; t < m; ++t) {
            const cpx w1 = tw[t * 3], w2 = tw[t * 3 + 1], w3 = tw[t * 3 + 2];
            for (int q = 0; q < s; ++q) {
                const cpx *a0p = x + (size_t)(q + s * t) * B, *a1p = x + (size_t)(q + s * (t + m)) * B;
                const cpx *a2p = x + (size_t)(q + s * (t + 2 * m)) * B, *a3p = x + (size_t)(q + s * (t + 3 * m)) * B;
                cpx *y0 = y + (size_t)(q + s * (4 * t)) * B, *y1 = y + (size_t)(q + s * (4 * t + 1)) * B;
                cpx *y2 = y + (size_t)(q + s * (4 * t + 2)) * B, *y3 = y + (size_t)(q + s * (4 * t + 3)) * B;
                for (int b = 0; b < B; ++b) {
                    cpx a0 = a0p[b], a1 = a1p[b], a2 = a2p[b], a3 = a3p[b];
                    float s02r = a0.r + a2.r, s02i = a0.i + a2.i, d02r = a0.r - a2.r, d02i = a0.i - a2.i;
                    float s13r = a1.r + a3.r, s13i = a1.i + a3.i, d13r = a1.r - a3.r, d13i = a1.i - a3.i;
                    float jr = -sg * d13i, ji = sg * d13r;
                    float b1r = d02r + jr, b1i = d02i + ji;
                    float b2r = s02r - s13r, b2i = s02i - s13i;
                    float b3r = d02r - jr, b3i = d02i - ji;
                    y0[b].r = s02r + s13r; y0[b].i = s02i + s13i;
                    y1[b].r = b1r * w1.r - b1i * w1.i; y1[b].i = b1r * w1.i + b1i * w1.r;
                    y2[b].r = b2r * w2.r - b2i * w2.i; y2[b].i = b2r * w2.i + b2i * w2.r;
                    y3[b].r = b3r * w3.r - b3i * w3.i; y3[b].i = b3r * w3.i + b3i * w3.r;
                }
            }
        }
    } else if (p == 3) {
        const float c = -0.5f;
        const float sn = sg * 0.86602540378443864676f;
        for (int t = 0; t < m; ++t) {
            const cpx w1 = tw[t * 2], w2 = tw[t * 2 + 1];
            for (int q = 0; q < s; ++q) {
                const cpx *a0p = x + (size_t)(q + s * t) * B, *a1p = x + (size_t)(q + s * (t + m)) * B;
                const cpx *a2p = x + (size_t)(q + s * (t + 2 * m)) * B;
                cpx *y0 = y + (size_t)(q + s * (3 * t)) * B, *y1 = y + (size_t)(q + s * (3 * t + 1)) * B;
                cpx *y2 = y + (size_t)(q + s * (3 * t + 2)) * B;
                for (int b = 0; b < B; ++b) {
                    cpx a0 = a0p[b], a1 = a1p[b], a2 = a2p[b];
                    float sr = a1.r + a2.r, si = a1.i + a2.i, dr = a1.r - a2.r, di = a1.i - a2.i;
                    float br = a0.r + c * sr, bi = a0.i + c * si;
                    float rr = -sn * di, ri = sn * dr;
                    float b1r = br + rr, b1i = bi + ri, b2r = br - rr, b2i = bi - ri;
                    y0[b].r = a0.r + sr; y0[b].i = a0.i + si;
                    y1[b].r = b1r * w1.r - b1i * w1.i; y1[b].i = b1r * w1.i + b1i * w1.r;
                    y2[b].r = b2r * w2.r - b2i * w2.i; y2[b].i = b2r * w2.i + b2i * w2.r;
                }
            }
        }
    } else if (p == 5) {
        /* DFT_5 with the usual symmetric split: c1=cos(2pi/5), c2=cos(4pi/5) */
        const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
        const float s1 = sg * 0.95105651629515357212f, s2 = sg * 0.58778525229247312917f;
        for (int t = 0; t < m; ++t) {
            const cpx w1 = tw[t * 4], w2 = tw[t * 4 + 1], w3 = tw[t * 4 + 2], w4 = tw[t * 4 + 3];
            for (int q = 0; q < s; ++q) {
                const cpx *ap[5];
                cpx *yp[5];
                for (int r = 0; r < 5; ++r) {
                    ap[r] = x + (size_t)(q + s * (t + r * m)) * B;
                    yp[r] = y + (size_t)(q + s * (5 * t + r)) * B;
                }
                for (int b = 0; b < B; ++b) {
                    cpx a0 = ap[0][b], a1 = ap[1][b], a2 = ap[2][b], a3 = ap[3][b], a4 = ap[4][b];
                    float p14r = a1.r + a4.r, p14i = a1.i + a4.i, m14r = a1.r - a4.r, m14i = a1.i - a4.i;
                    float p23r = a2.r + a3.r, p23i = a2.i + a3.i, m23r = a2.r - a3.r, m23i = a2.i - a3.i;
                    float tAr = a0.r + c1 * p14r + c2 * p23r, tAi = a0.i + c1 * p14i + c2 * p23i;
                    float tBr = a0.r + c2 * p14r + c1 * p23r, tBi = a0.i + c2 * p14i + c1 * p23i;
                    /* i*(s1*m14 + s2*m23) and i*(s2*m14 - s1*m23) */
                    float uAr = -(s1 * m14i + s2 * m23i), uAi = s1 * m14r + s2 * m23r;
                    float uBr = -(s2 * m14i - s1 * m23i), uBi = s2 * m14r - s1 * m23r;
                    float b1r = tAr + uAr, b1i = tAi + uAi, b4r = tAr - uAr, b4i = tAi - uAi;
                    float b2r = tBr + uBr, b2i = tBi + uBi, b3r = tBr - uBr, b3i = tBi - uBi;
                    yp[0][b].r = a0.r + p14r + p23r; yp[0][b].i = a0.i + p14i + p23i;
                    yp[1][b].r = b1r * w1.r - b1i * w1.i; yp[1][b].i = b1r * w1.i + b1i * w1.r;
                    yp[2][b].r = b2r * w2.r - b2i * w2.i; yp[2][b].i = b2r * w2.i + b2i * w2.r;
                    yp[3][b].r = b3r * w3.r - b3i * w3.i; yp[3][b].i = b3r * w3.i + b3i * w3.r;
                    yp[4][b].r = b4r * w4.r - b4i * w4.i; yp[4][b].i = b4r * w4.i + b4i * w4.r;
                }
            }
        }
    } else {
        const cpx *W = pl->wp[st];
        for (int t = 0; t < m; ++t)
            for (int q = 0; q < s; ++q)
                for (int b = 0; b < B; ++b)
                    for (int k = 0; k < p; ++k) {
                        float br = 0.f, bi = 0.f;
                        for (int r = 0; r < p; ++r) {
                            cpx a = x[(size_t)(q + s * (t + r * m)) * B + b];
                            cpx w = W[k * p + r];
                            br += a.r * w.r - a.i * w.i;
                            bi += a.r * w.i + a.i * w.r;
                        }
                        cpx out = {br, bi};
                        if (k) {
                            cpx w = tw[t * (p - 1) + (k - 1)];
                            out.r = br * w.r - bi * w.i;
                            out.i = br * w.i + bi * w.r;
                        }
                        y[(size_t)(q + s * (p * t + k)) * B + b] = out;
                    }
    }
}

/* In-place batched transform: data holds B vectors of length pl->n laid out
 * as data[j*B + b]; work must hold n*B elements. */
static void cfft_batch(const cplan *pl, cpx *data, int B, cpx *work) {
    int n = pl->n;
    if (n <= 1) return;
    cpx *x = data, *y = work;
    int len = n, s = 1;
    for (int st = 0; st < pl->nstage; ++st) {
        stage(pl, st, len, s, B, x, y);
        len /= pl->radix[st];
        s *= pl->radix[st];
        cpx *tmp = x; x = y; y = tmp;
    }
    if (x != data) memcpy(data, x, sizeof(cpx) * (size_t)n * B);
}

/* single contiguous vector */
static void cfft_exec(cplan *pl, cpx *data) { cfft_batch(pl, data, 1, pl->bufa); }

/* ------------------------------------------------------------------ */
/* Real transforms along the last (contiguous) dimension, in row blocks */
/* ------------------------------------------------------------------ */
#define ROWBLOCK 16

typedef struct {
    int n;
    int even;
    cplan half;      /* length n/2 when even, n otherwise */
    cpx *split;      /* exp(sign*2*pi*i*k/n), k in [0, n/2] */
    cpx *z, *work;   /* batched buffers: (n or n/2) * ROWBLOCK */
} rplan;

static void rplan_init(rplan *rp, int n, int sign) {
    rp->n = n;
    rp->even = (n % 2 == 0) && n >= 2;
    int hl = rp->even ? n / 2 : n;
    cplan_init(&rp->half, hl, sign);
    rp->split = (cpx *)malloc(sizeof(cpx) * (size_t)(n / 2 + 1));
    for (int k = 0; k <= n / 2; ++k) {
        double ang = sign * 2.0 * M_PI * (double)k / (double)n;
        rp->split[k].r = (float)cos(ang);
        rp->split[k].i = (float)sin(ang);
    }
    rp->z = (cpx *)malloc(sizeof(cpx) * (size_t)(hl > 0 ? hl : 1) * ROWBLOCK);
    rp->work = (cpx *)malloc(sizeof(cpx) * (size_t)(hl > 0 ? hl : 1) * ROWBLOCK);
}

static void rplan_free(rplan *rp) {
    cplan_free(&rp->half);
    free(rp->split);
    free(rp->z);
    free(rp->work);
}

/* forward real transforms of R rows: in[r*nx + j] -> out[r*hx + k] */
static void r2c_rows(rplan *rp, const float *in, cpx *out, int R, int nx, int hx) {
    const int n = rp->n;
    cpx *z = rp->z;
    if (!rp->even) {
        for (int j = 0; j < n; ++j)
            for (int r = 0; r < R; ++r) { z[(size_t)j * R + r].r = in[(size_t)r * nx + j]; z[(size_t)j * R + r].i = 0.f; }
        cfft_batch(&rp->half, z, R, rp->work);
        for (int k = 0; k <= n / 2; ++k)
            for (int r = 0; r < R; ++r) out[(size_t)r * hx + k] = z[(size_t)k * R + r];
        return;
    }
    const int h = n / 2;
    for (int j = 0; j < h; ++j)
        for (int r = 0; r < R; ++r) {
            z[(size_t)j * R + r].r = in[(size_t)r * nx + 2 * j];
            z[(size_t)j * R + r].i = in[(size_t)r * nx + 2 * j + 1];
        }
    cfft_batch(&rp->half, z, R, rp->work);
    for (int k = 0; k <= h; ++k) {
        const cpx w = rp->split[k];
        const cpx *zk = z + (size_t)(k % h) * R, *zc = z + (size_t)((h - k) % h) * R;
        for (int r = 0; r < R; ++r) {
            float er = 0.5f * (zk[r].r + zc[r].r), ei = 0.5f * (zk[r].i - zc[r].i);
            float dr = 0.5f * (zk[r].r - zc[r].r), di = 0.5f * (zk[r].i + zc[r].i);
            /* O*w^k = (-i*d)*w with d = Z[k]-conj(Z[h-k]) over 2 */
            float orr = di, oi = -dr;
            out[(size_t)r * hx + k].r = er + orr * w.r - oi * w.i;
            out[(size_t)r * hx + k].i = ei + orr * w.i + oi * w.r;
        }
    }
}

/* inverse real transforms (unnormalised) of R rows: in[r*hx + k] -> out[r*nx + j] */
static void c2r_rows(rplan *rp, const cpx *in, float *out, int R, int nx, int hx) {
    const int n = rp->n;
    cpx *z = rp->z;
    if (!rp->even) {
        for (int k = 0; k < n; ++k)
            for (int r = 0; r < R; ++r) {
                cpx v;
                if (k <= n / 2) v = in[(size_t)r * hx + k];
                else { v = in[(size_t)r * hx + (n - k)]; v.i = -v.i; }
                if (k == 0) v.i = 0.f;
                z[(size_t)k * R + r] = v;
            }
        cfft_batch(&rp->half, z, R, rp->work);
        for (int j = 0; j < n; ++j)
            for (int r = 0; r < R; ++r) out[(size_t)r * nx + j] = z[(size_t)j * R + r].r;
        return;
    }
    const int h = n / 2;
    for (int k = 0; k < h; ++k) {
        const cpx w = rp->split[k];
        for (int r = 0; r < R; ++r) {
            cpx xk = in[(size_t)r * hx + k], xc = in[(size_t)r * hx + (h - k)];
            if (k == 0) { xk.i = 0.f; xc.i = 0.f; }
            float sr = xk.r + xc.r, si = xk.i - xc.i;
            float dr = xk.r - xc.r, di = xk.i + xc.i;
            float dwr = dr * w.r - di * w.i, dwi = dr * w.i + di * w.r;
            z[(size_t)k * R + r].r = sr - dwi;
            z[(size_t)k * R + r].i = si + dwr;
        }
    }
    cfft_batch(&rp->half, z, R, rp->work);
    for (int j = 0; j < h; ++j)
        for (int r = 0; r < R; ++r) {
            out[(size_t)r * nx + 2 * j] = z[(size_t)j * R + r].r;
            out[(size_t)r * nx + 2 * j + 1] = z[(size_t)j * R + r].i;
        }
}

/* ------------------------------------------------------------------ */
/* FFTW-style plans                                                     */
/* ------------------------------------------------------------------ */
enum { K_R2C = 1, K_C2R = 2, K_MANY = 3 };

struct g2s_shim_plan_s {
    int kind;
    int rank;
    int n[8];
    float *rin;
    cpx *cin;
    float *rout;
    cpx *cout;
    int howmany, istride, idist, ostride, odist;
    rplan row;            /* last dimension (r2c/c2r) */
    cplan dim[8];         /* complex plans for dims 0..rank-2 (or dim 0 for many) */
    cpx *colwork;         /* work buffer for batched strided transforms */
    cpx *colbuf;          /* gather buffer (many-dft) */
};

#define COLBLOCK 16

static int prod(const int *n, int a, int b) {
    int r = 1;
    for (int i = a; i < b; ++i) r *= n[i];
    return r;
}

/* complex FFT along dimension d of a row-major complex array: every slice
 * [nd][inner] is already in batched layout with batch = inner. */
static void fft_along(struct g2s_shim_plan_s *p, cpx *a, const int *shape, int rank, int d) {
    const int nd = shape[d];
    const int inner = prod(shape, d + 1, rank);
    const int outer = prod(shape, 0, d);
    for (int o = 0; o < outer; ++o)
        cfft_batch(&p->dim[d], a + (size_t)o * nd * inner, inner, p->colwork);
}

static struct g2s_shim_plan_s *plan_rc(int kind, int rank, const int *n) {
    if (rank < 1 || rank > 8) return NULL;
    struct g2s_shim_plan_s *p = (struct g2s_shim_plan_s *)calloc(1, sizeof(*p));
    p->kind = kind;
    p->rank = rank;
    for (int i = 0; i < rank; ++i) p->n[i] = n[i];
    int sign = (kind == K_R2C) ? FFTW_FORWARD : FFTW_BACKWARD;
    rplan_init(&p->row, n[rank - 1], sign);
    for (int d = 0; d < rank - 1; ++d) cplan_init(&p->dim[d], n[d], sign);
    size_t half = (size_t)prod(n, 0, rank - 1) * (size_t)(n[rank - 1] / 2 + 1);
    p->colwork = (cpx *)malloc(sizeof(cpx) * (half > 0 ? half : 1));
    return p;
}

fftwf_plan fftwf_plan_dft_r2c(int rank, const int *n, float *in, fftwf_complex *out, unsigned flags) {
    (void)flags;
    struct g2s_shim_plan_s *p = plan_rc(K_R2C, rank, n);
    if (!p) return NULL;
    p->rin = in;
    p->cout = (cpx *)out;
    return p;
}

fftwf_plan fftwf_plan_dft_c2r(int rank, const int *n, fftwf_complex *in, float *out, unsigned flags) {
    (void)flags;
    struct g2s_shim_plan_s *p = plan_rc(K_C2R, rank, n);
    if (!p) return NULL;
    p->cin = (cpx *)in;
    p->rout = out;
    return p;
}

fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany,
                               fftwf_complex *in, const int *inembed, int istride, int idist,
                               fftwf_complex *out, const int *onembed, int ostride, int odist,
                               int sign, unsigned flags) {
    (void)inembed; (void)onembed; (void)flags;
    if (rank != 1) return NULL; /* only the rank-1 form is used by the G2S CPU device */
    struct g2s_shim_plan_s *p = (struct g2s_shim_plan_s *)calloc(1, sizeof(*p));
    p->kind = K_MANY;
    p->rank = 1;
    p->n[0] = n[0];
    p->cin = (cpx *)in;
    p->cout = (cpx *)out;
    p->howmany = howmany;
    p->istride = istride; p->idist = idist;
    p->ostride = ostride; p->odist = odist;
    cplan_init(&p->dim[0], n[0], sign);
    p->colbuf = (cpx *)malloc(sizeof(cpx) * (size_t)n[0] * COLBLOCK);
    p->colwork = (cpx *)malloc(sizeof(cpx) * (size_t)n[0] * COLBLOCK);
    return p;
}

static void exec_r2c(struct g2s_shim_plan_s *p, float *in, cpx *out) {
    const int rank = p->rank;
    const int nx = p->n[rank - 1];
    const int hx = nx / 2 + 1;
    const int rows = prod(p->n, 0, rank - 1);
    for (int r0 = 0; r0 < rows; r0 += ROWBLOCK) {
        int R = rows - r0 < ROWBLOCK ? rows - r0 : ROWBLOCK;
        r2c_rows(&p->row, in + (size_t)r0 * nx, out + (size_t)r0 * hx, R, nx, hx);
    }
    int shape[8] = {0};
    for (int i = 0; i < rank && i < 8; ++i) shape[i] = p->n[i];
    shape[rank - 1] = hx;
    for (int d = rank - 2; d >= 0; --d) fft_along(p, out, shape, rank, d);
}

static void exec_c2r(struct g2s_shim_plan_s *p, cpx *in, float *out) {
    const int rank = p->rank;
    const int nx = p->n[rank - 1];
    const int hx = nx / 2 + 1;
    const int rows = prod(p->n, 0, rank - 1);
    int shape[8] = {0};
    for (int i = 0; i < rank && i < 8; ++i) shape[i] = p->n[i];
    shape[rank - 1] = hx;
    /* like FFTW's default for c2r, the input array is overwritten */
    for (int d = 0; d <= rank - 2; ++d) fft_along(p, in, shape, rank, d);
    for (int r0 = 0; r0 < rows; r0 += ROWBLOCK) {
        int R = rows - r0 < ROWBLOCK ? rows - r0 : ROWBLOCK;
        c2r_rows(&p->row, in + (size_t)r0 * hx, out + (size_t)r0 * nx, R, nx, hx);
    }
}

static void exec_many(struct g2s_shim_plan_s *p) {
    const int n0 = p->n[0];
    for (int v0 = 0; v0 < p->howmany; v0 += COLBLOCK) {
        int vb = p->howmany - v0 < COLBLOCK ? p->howmany - v0 : COLBLOCK;
        for (int j = 0; j < n0; ++j)
            for (int v = 0; v < vb; ++v)
                p->colbuf[(size_t)j * vb + v] = p->cin[(size_t)(v0 + v) * p->idist + (size_t)j * p->istride];
        cfft_batch(&p->dim[0], p->colbuf, vb, p->colwork);
        for (int j = 0; j < n0; ++j)
            for (int v = 0; v < vb; ++v)
                p->cout[(size_t)(v0 + v) * p->odist + (size_t)j * p->ostride] = p->colbuf[(size_t)j * vb + v];
    }
}

void fftwf_execute(const fftwf_plan p) {
    if (!p) return;
    switch (p->kind) {
    case K_R2C: exec_r2c(p, p->rin, p->cout); break;
    case K_C2R: exec_c2r(p, p->cin, p->rout); break;
    case K_MANY: exec_many(p); break;
    }
}

void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out) {
    if (p && p->kind == K_C2R) exec_c2r(p, (cpx *)in, out);
}

void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out) {
    if (p && p->kind == K_R2C) exec_r2c(p, in, (cpx *)out);
}

void fftwf_destroy_plan(fftwf_plan p) {
    if (!p) return;
    if (p->kind == K_R2C || p->kind == K_C2R) {
        rplan_free(&p->row);
        for (int d = 0; d < p->rank - 1; ++d) cplan_free(&p->dim[d]);
    } else {
        cplan_free(&p->dim[0]);
    }
    free(p->colwork);
    free(p->colbuf);
    free(p);
}

void fftwf_plan_with_nthreads(int nthreads) { (void)nthreads; }
int fftwf_init_threads(void) { return 1; }
void fftwf_cleanup_threads(void) {}
