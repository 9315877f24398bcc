/*
 * spmv_oracle.c -- ORACLE TEST INFRASTRUCTURE: plain-C restatement of the reference's
 * hot path (see spmv_oracle.h).  Used only as the checker (tests/, smoke check, the
 * bench's CPU-baseline leg).  Every function names the reference lines it restates.
 *
 * The converters are restated from the layout *definitions* (closed-form slot positions)
 * rather than from the reference's incremental pointer walks, so that agreeing with the
 * reference's own compiled converters is a real cross-check of both.
 */
#include "spmv_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static u32 cdiv(u32 a, u32 b) { return (a + b - 1) / b; }

/* ------------------------------------------------------------------ CSR */

/* cudaSpmv.cu:451-466: y[i] = ((0 + v0*x0) + v1*x1) + ... in CSR order, separate mul/add. */
void orc_csr_spmv(u32 n, const u32 *row, const u32 *col, const double *val, const double *x,
                  double *y)
{
    for (u32 i = 0; i < n; i++) {
        double acc = 0.0;
        for (u32 j = row[i]; j < row[i + 1]; j++) {
            double p = val[j] * x[col[j]];
            acc = acc + p;
        }
        y[i] = acc;
    }
}

void orc_csr_spmv_truth(u32 n, const u32 *row, const u32 *col, const double *val,
                        const double *x, double *y_true, double *abs_ax)
{
    for (u32 i = 0; i < n; i++) {
        long double acc = 0.0L;
        double mag = 0.0;
        for (u32 j = row[i]; j < row[i + 1]; j++) {
            acc += (long double)val[j] * (long double)x[col[j]];
            mag += fabs(val[j]) * fabs(x[col[j]]);
        }
        y_true[i] = (double)acc;
        abs_ax[i] = mag;
    }
}

void orc_csr_spmm(u32 n, u32 k, const u32 *row, const u32 *col, const double *val,
                  const double *X, double *Y)
{
    for (u32 i = 0; i < n; i++) {
        for (u32 q = 0; q < k; q++) Y[(size_t)i * k + q] = 0.0;
        for (u32 j = row[i]; j < row[i + 1]; j++)
            for (u32 q = 0; q < k; q++)
                Y[(size_t)i * k + q] += val[j] * X[(size_t)col[j] * k + q];
    }
}

/* cudaSpmv.cu:332-358.  rave2 accumulates rl*rl computed in 32-bit unsigned arithmetic,
 * exactly as the reference does (it wraps for rows longer than 65535). */
void orc_row_stats(u32 n, const u32 *row, const u32 *col, u32 *rl, double *out5)
{
    u32 rmin = 1000000000u, rmax = 0, bw = 0;
    double s1 = 0.0, s2 = 0.0;
    for (u32 i = 0; i < n; i++) {
        u32 l = row[i + 1] - row[i];
        rl[i] = l;
        s1 += l;
        s2 += (double)(u32)(l * l);
        if (l < rmin) rmin = l;
        if (l > rmax) rmax = l;
        for (u32 j = row[i]; j < row[i + 1]; j++) {
            int d = abs((int)i - (int)col[j]);
            if ((u32)d > bw) bw = (u32)d;
        }
    }
    s1 /= (double)n;
    s2 /= (double)n;
    out5[0] = rmin;
    out5[1] = s1;
    out5[2] = rmax;
    out5[3] = sqrt(s2 - s1 * s1);
    out5[4] = bw;
}

/* cudaSpmv.cu:474-495: max | |ac| - |ar| |, that over max|ar|, first argmax. */
void orc_get_errors(u32 n, const double *ar, const double *ac, double *aErr, double *rErr,
                    u32 *pos)
{
    double md = 0.0, mv = 0.0;
    u32 p = 0;
    for (u32 i = 0; i < n; i++) {
        double v = fabs(ar[i]);
        if (v > mv) mv = v;
        double d = fabs(fabs(ac[i]) - v);
        if (d > md) { md = d; p = i; }
    }
    *aErr = md;
    *rErr = md / mv;
    *pos = p;
}

/* ------------------------------------------------------------------ K1 */

u32 orc_k1_chunknum(u32 n) { return cdiv(n, 32); }

/* Stable merge sort of row indices by descending length: ties keep ascending row index,
 * which is what glibc's (mergesort-based) qsort gives for orderFunction
 * (cudaSpmv.cu:716-737). */
static void msort_desc(u32 *idx, u32 *tmp, const u32 *key, u32 lo, u32 hi)
{
    if (hi - lo < 2) return;
    u32 mid = lo + (hi - lo) / 2;
    msort_desc(idx, tmp, key, lo, mid);
    msort_desc(idx, tmp, key, mid, hi);
    u32 a = lo, b = mid, o = lo;
    while (a < mid && b < hi) {
        /* take from the right run only when strictly longer: keeps stability */
        if (key[idx[b]] > key[idx[a]]) tmp[o++] = idx[b++];
        else tmp[o++] = idx[a++];
    }
    while (a < mid) tmp[o++] = idx[a++];
    while (b < hi) tmp[o++] = idx[b++];
    memcpy(idx + lo, tmp + lo, (size_t)(hi - lo) * sizeof(u32));
}

void orc_k1_perm(u32 n, const u32 *rl, u32 *permi)
{
    u32 *tmp = (u32 *)malloc((size_t)(n ? n : 1) * sizeof(u32));
    for (u32 i = 0; i < n; i++) permi[i] = i;
    msort_desc(permi, tmp, rl, 0, n);
    free(tmp);
}

/* cudaSpmv.cu:741-754: nmc = length of each chunk's first (longest) row; chp = exclusive
 * prefix of 32*nmc; lenVC = total. */
u32 orc_k1_nmc_chp(u32 n, const u32 *rl, const u32 *permi, u32 *nmc, u32 *chp)
{
    u32 nc = orc_k1_chunknum(n), len = 0;
    for (u32 c = 0; c < nc; c++) {
        nmc[c] = rl[permi[c * 32]];
        chp[c] = len;
        len += 32 * nmc[c];
    }
    return len;
}

/* cudaSpmv.cu:758-778: element j of sorted row 32c+l lands at chp[c] + 32j + l. */
void orc_k1_fill(u32 n, const u32 *row, const u32 *col, const double *val, const u32 *permi,
                 const u32 *chp, double *kval, u32 *kcol)
{
    for (u32 g = 0; g < n; g++) {
        u32 r = permi[g], c = g / 32, l = g % 32;
        for (u32 j = 0; j < row[r + 1] - row[r]; j++) {
            u32 pos = chp[c] + 32 * j + l;
            kval[pos] = val[row[r] + j];
            kcol[pos] = col[row[r] + j];
        }
    }
}

/* gk1 (cudaSpmv.cu:851-867): sum over the chunk's nmc stored slots of each sorted row,
 * stored padding included; y scattered through permi.  Empty chunks read nothing. */
void orc_k1_spmv(u32 n, const u32 *permi, const u32 *nmc, const u32 *chp, const double *kval,
                 const u32 *kcol, const double *x, double *y)
{
    for (u32 g = 0; g < n; g++) {
        u32 c = g / 32, l = g % 32;
        double acc = 0.0;
        for (u32 j = 0; j < nmc[c]; j++) {
            u32 pos = chp[c] + 32 * j + l;
            double p = kval[pos] * x[kcol[pos]];
            acc = acc + p;
        }
        y[permi[g]] = acc;
    }
}

/* ------------------------------------------------------------------ AXC */

/* cudaSpmv.cu:937-948: brp[r+1] = brp[r] + 2*hbs*ceil(rl/hbs). */
u32 orc_axc_brp(u32 n, u32 hbs, const u32 *rl, u32 *brp)
{
    brp[0] = 0;
    for (u32 r = 0; r < n; r++) brp[r + 1] = brp[r] + 2 * hbs * cdiv(rl[r], hbs);
    return brp[n];
}

/* cudaSpmv.cu:952-999: element j of row r sits in brick j/hbs of the row, lane j%hbs;
 * mapx lists the row's columns compactly from brp[r]/2. */
void orc_axc_fill(u32 n, u32 hbs, const u32 *row, const u32 *col, const double *val,
                  const double *x, const u32 *brp, double *ax, double *nval, u32 *ncol,
                  u32 *mapx)
{
    for (u32 r = 0; r < n; r++) {
        u32 s0 = brp[r] / 2;
        for (u32 j = 0; j < row[r + 1] - row[r]; j++) {
            u32 p = row[r] + j, s = s0 + j;
            u32 a = (s / hbs) * 2 * hbs + s % hbs;
            if (ax) { ax[a] = val[p]; ax[a + hbs] = x[col[p]]; }
            if (nval) { nval[s] = val[p]; ncol[s] = col[p]; }
            if (mapx) mapx[s] = col[p];
        }
    }
}

/* ------------------------------------------------------------------ AXT */

/* the reference's integer log loops: logTH (cudaSpmv.cu:1404-1405), log for COM
 * (cudaSpmv.cu:1504-1511 with bs, 1529-1536 with th). */
static u32 ilog_loop(u32 v, u32 from, u32 to_excl, u32 dflt)
{
    for (u32 i = from; i < to_excl; i++)
        if ((v >> i) == 1) return i;
    return dflt;
}

int orc_axt_dims_con(u32 n, const u32 *rl, u32 thw, u32 th, u32 bs, int mode, u32 *con,
                     orc_axt_dims *d)
{
    if (thw == 0 || th == 0) return -1;
    const u32 ths = thw * th;
    memset(d, 0, sizeof(*d));
    d->lenCON = n;
    d->logTH = ilog_loop(th, 0, 10, 0);
    if (mode == 0 && th == 1) {
        /* cudaSpmv.cu:1158-1175: each row gets ceil(rl/thw) whole tiles */
        u32 tiles = 0;
        con[0] = 0;
        for (u32 r = 0; r < n; r++) {
            u32 t = cdiv(rl[r], thw);
            tiles += t;
            con[r + 1] = con[r] + t * 2 * thw;
        }
        d->tileN = tiles;
        d->lenAX = tiles * 2 * thw;
        d->lenSEC = tiles;
    } else if (mode == 0) {
        /* cudaSpmv.cu:1179-1201: rows padded to a multiple of th; a row starts at tile
         * column C = (start position)/th, i.e. ax index (C/thw)*2*ths + C%thw. */
        u32 cols = 0;
        for (u32 r = 0; r < n; r++) {
            u32 t = cols / thw, c = cols % thw;
            con[r] = t * 2 * ths + c;
            cols += cdiv(rl[r], th);
        }
        d->tileN = cdiv(cols, thw);
        d->lenAX = d->tileN * 2 * ths;
        d->lenSEC = d->tileN * thw;
    } else {
        /* cudaSpmv.cu:1205-1235: no per-row padding, only the last tile is padded */
        u32 tot = 0;
        for (u32 r = 0; r < n; r++) tot += rl[r];
        u32 w = (th == 1) ? thw : ths;
        d->tileN = cdiv(tot, w);
        d->lenAX = 2 * d->tileN * w;
        d->lenSEC = d->tileN * w;
        d->log = (th == 1) ? ilog_loop(bs, 1, 11, 0) : ilog_loop(th, 1, 10, 0);
    }
    return 0;
}

/* slot of CSR position p of a COM layout; its ax index is (slot/thw)*2*thw + slot%thw */
static u32 com_slot(u32 p, u32 thw, u32 th)
{
    if (th == 1) return p;
    u32 ths = thw * th, t = p / ths, f = p % th, c = (p - t * ths) / th;
    return t * ths + f * thw + c;
}

void orc_axt_fill(u32 n, const u32 *row, const u32 *col, const double *val, const double *x,
                  u32 thw, u32 th, u32 bs, int mode, const u32 *con, const orc_axt_dims *d,
                  double *ax, double *nval, u32 *ncol, u32 *sec)
{
    const u32 ths = thw * th;
    for (u32 r = 0; r < n; r++) {
        u32 len = row[r + 1] - row[r];
        for (u32 e = 0; e < len; e++) {
            u32 p = row[r] + e, s;
            if (mode == 0 && th == 1) {
                /* cudaSpmv.cu:1239-1271: slot = row's first slot + e; sec per tile */
                s = con[r] / 2 + e;
                sec[s / thw] = r;
            } else if (mode == 0) {
                /* cudaSpmv.cu:1275-1308: element e in column C_r + e/th, tile row e%th */
                u32 c0 = (con[r] / (2 * ths)) * thw + con[r] % thw;
                u32 C = c0 + e / th, f = e % th;
                s = (C / thw) * ths + f * thw + C % thw;
                sec[(C / thw) * thw + C % thw] = r;
            } else {
                /* cudaSpmv.cu:1312-1387: headers (row << log) | remaining-in-segment at a
                 * row start and at every segment boundary (bs block for th=1, tile column
                 * start for th>1); other slots keep sec = 0 */
                s = com_slot(p, thw, th);
                u32 f = (th == 1) ? p % bs : p % th;
                u32 lim = (th == 1) ? bs - 1 - f : th - 1 - f;
                if (e == 0 || f == 0) {
                    u32 q1 = len - e - 1;
                    sec[s] = (r << d->log) | (q1 > lim ? lim : q1);
                }
            }
            u32 a = (s / thw) * 2 * thw + s % thw;
            if (ax) { ax[a] = val[p]; ax[a + thw] = x[col[p]]; }
            if (nval) { nval[s] = val[p]; ncol[s] = col[p]; }
        }
    }
}

/* Segment walk over a COM header stream: the segment starting at CSR position p covers
 * positions p..p+offset of row (hdr >> log).  Only power-of-two bs (th=1) / th (th>1)
 * decode unambiguously. */
static int com_walk(u32 n, u32 nnz_slots, u32 thw, u32 th, u32 bs, u32 log, const u32 *sec,
                    const double *vals, const u32 *cols, const double *x, const double *ax,
                    double *y)
{
    u32 blk = (th == 1) ? bs : th;
    if (blk == 0 || (blk & (blk - 1)) != 0 || (1u << log) != blk) return -1;
    u32 mask = blk - 1;
    for (u32 p = 0; p < nnz_slots;) {
        u32 s = com_slot(p, thw, th);
        u32 h = sec[s], r = h >> log, o = h & mask;
        if (r >= n) return -1;
        double acc = 0.0;
        for (u32 q = p; q <= p + o; q++) {
            u32 sq = com_slot(q, thw, th);
            double xv;
            double v;
            if (ax) {
                u32 a = (sq / thw) * 2 * thw + sq % thw;
                v = ax[a];
                xv = ax[a + thw];
            } else {
                v = vals[sq];
                xv = x[cols[sq]];
            }
            acc = acc + v * xv;
        }
        y[r] += acc;
        p += o + 1;
    }
    return 0;
}

static int axt_spmv_any(u32 n, u32 thw, u32 th, u32 bs, int mode, const orc_axt_dims *d,
                        const u32 *sec, const double *nval, const u32 *ncol, const double *x,
                        const double *ax, double *y, u32 nnz)
{
    const u32 ths = thw * th;
    for (u32 i = 0; i < n; i++) y[i] = 0.0;
    if (mode != 0) return com_walk(n, nnz, thw, th, bs, d->log, sec, nval, ncol, x, ax, y);
    for (u32 t = 0; t < d->tileN; t++) {
        for (u32 c = 0; c < thw; c++) {
            u32 r = (th == 1) ? sec[t] : sec[t * thw + c];
            if (r >= n) return -1;
            double acc = 0.0;
            for (u32 f = 0; f < th; f++) {
                u32 s = t * ths + f * thw + c;
                double v, xv;
                if (ax) {
                    u32 a = (s / thw) * 2 * thw + s % thw;
                    v = ax[a];
                    xv = ax[a + thw];
                } else {
                    v = nval[s];
                    xv = x[ncol[s]];
                }
                acc = acc + v * xv;
            }
            y[r] += acc;
        }
    }
    return 0;
}

int orc_axt_spmv(u32 n, u32 thw, u32 th, u32 bs, int mode, const orc_axt_dims *d,
                 const u32 *sec, const double *nval, const u32 *ncol, const double *x,
                 double *y)
{
    /* COM layouts hold nnz real slots in CSR order; count them from the headers' extent */
    u32 nnz = 0;
    if (mode != 0) {
        /* the last tile's padding has sec == 0 after the last segment: walk until the
         * header stream runs past the data, which the caller bounds with lenSEC */
        nnz = d->lenSEC;
    }
    return axt_spmv_any(n, thw, th, bs, mode, d, sec, nval, ncol, x, NULL, y, nnz);
}

int orc_axt_spmv_baked(u32 n, u32 thw, u32 th, u32 bs, int mode, const orc_axt_dims *d,
                       const u32 *sec, const double *ax, double *y)
{
    u32 nnz = (mode != 0) ? d->lenSEC : 0;
    return axt_spmv_any(n, thw, th, bs, mode, d, sec, NULL, NULL, NULL, ax, y, nnz);
}
