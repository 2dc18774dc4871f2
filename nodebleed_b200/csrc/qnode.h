// Encoding of one 8-wide node in the GPU layout (gpulayout.h), shared by the
// host conversion of the reference BVH8 (layout.cpp) and the device TLAS
// build (tlas_build.cuh), so both produce the same bytes for the same child
// boxes: the greedy slot assignment and the conservative 8-bit quantisation.
// Every operation is an IEEE-754 operation with one rounding, with no fused
// multiply-add (the host file is built without FMA, the device file with
// -fmad=false), so host and device results are identical.

#ifndef NB_QNODE_H
#define NB_QNODE_H

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "gpulayout.h"

#ifdef __CUDACC__
#define NB_HD __host__ __device__
#else
#define NB_HD
#endif

namespace nb {

// ceil(log2(x)) for a finite x > 0, exactly (frexp is exact: x = m 2^k with
// m in [0.5, 1); x is a power of two iff m = 0.5).
NB_HD inline int ceil_log2(double x)
{
	int k = 0;
	double m = frexp(x, &k);
	return m == 0.5 ? k - 1 : k;
}

// Greedy assignment of children to slots: slot s prefers children lying
// towards (+/-x, +/-y, +/-z) by its bits, so that ascending slot ^ octant is
// roughly near-to-far for rays of that octant (after Ylitie, Karras and
// Laine 2017).  cen: child box centres, nc: node box centre.  A round in
// which no score beats -FLT_MAX (NaN or -inf scores, from centres that
// overflowed) takes the first free (child, slot) pair, so every child gets
// a slot.
NB_HD inline void assign_slots(int nchild, const float cen[8][3],
                               const float nc[3], int slot_of[8])
{
	bool used_c[8] = {false, false, false, false, false, false, false,
	  false};
	bool used_s[8] = {false, false, false, false, false, false, false,
	  false};
	for (int i = 0; i < 8; i++)
		slot_of[i] = -1;
	for (int round = 0; round < nchild; round++) {
		float best = -FLT_MAX;
		int bc = -1, bs = -1, fc = -1, fs = -1;
		for (int c = 0; c < nchild; c++) {
			if (used_c[c])
				continue;
			for (int s = 0; s < 8; s++) {
				if (used_s[s])
					continue;
				if (fc < 0) {
					fc = c;
					fs = s;
				}
				float sc = 0.0f;
				for (int a = 0; a < 3; a++)
					sc += (cen[c][a] - nc[a]) *
					  ((s >> a) & 1 ? 1.0f : -1.0f);
				if (sc > best) {
					best = sc;
					bc = c;
					bs = s;
				}
			}
		}
		if (bc < 0) {
			bc = fc;
			bs = fs;
		}
		used_c[bc] = used_s[bs] = true;
		slot_of[bc] = bs;
	}
}

// Stored exponent byte of a scale 2^e.  The device forms 2^(byte - 127) =
// 2^(e - 8), the scale of a plane byte placed in bits 8..15 of the float
// 2^23 + 256 q (trace.cuh: visit).
constexpr int kQExpBias = 127 - 8;

// Margin, in quanta, by which child planes are rounded outwards beyond the
// exact child box.  It covers the absolute rounding error of the device's
// plane distances, at most 2^-9 + 2^-14 quanta (trace.cuh: visit); errors
// relative to the distance are covered there by widening the far plane.
constexpr double kQMargin = 1.0 / 32.0;

// Bound on the node frame's coordinates: infinite child bounds (a transform
// that overflows float, vertices next to FLT_MAX) are clamped to +-2^125 for
// the origin and exponent, so the exponent search always ends with a finite
// origin.  Child planes beyond the frame saturate at 0 and 255: geometry
// farther out than 2^125 (4.25e37) need not lie inside its box.
constexpr float kQFrameMax = 4.2535296e37f; // 2^125

// Quantise one node: child boxes (min/max per slot; empty slots have
// min > max) into n's origin, exponents and qlo/qhi.  Per axis the scale is
// the smallest power of two 2^e with the node box spanning at most 249
// quanta (and at least 2^-22 of the coordinates' magnitude); the origin
// lies two quanta below the box, rounded down to a float; child planes are
// rounded outwards from the child box widened by kQMargin quanta.  Other
// fields of n are left as they are.
NB_HD inline void quantise_node_hd(const float cmin[8][3],
                                   const float cmax[8][3], nb_qnode *n)
{
	float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
	float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
	bool any = false;
	for (int s = 0; s < 8; s++) {
		if (!(cmin[s][0] <= cmax[s][0] && cmin[s][1] <= cmax[s][1] &&
		  cmin[s][2] <= cmax[s][2]))
			continue;
		any = true;
		for (int a = 0; a < 3; a++) {
			lo[a] = fminf(lo[a], cmin[s][a]);
			hi[a] = fmaxf(hi[a], cmax[s][a]);
		}
	}
	if (!any)
		for (int a = 0; a < 3; a++)
			lo[a] = hi[a] = 0.0f;
	for (int a = 0; a < 3; a++) {
		lo[a] = fminf(fmaxf(lo[a], -kQFrameMax), kQFrameMax);
		hi[a] = fminf(fmaxf(hi[a], -kQFrameMax), kQFrameMax);
	}
	float p[3];
	int ex[3];
	for (int a = 0; a < 3; a++) {
		double ext = (double)hi[a] - lo[a];
		double floor_scale = fmax(fabs((double)lo[a]),
		  fabs((double)hi[a])) * ldexp(1.0, -22);
		double need = fmax(fmax(ext / 249.0, floor_scale), ldexp(1.0, -100));
		int e = ceil_log2(need);
		// ends by e = 254 - kQExpBias at the latest, whatever the input;
		// the frame bound keeps it far below that
		for (;; e++) {
			// a power of two: multiplying by 2^-e divides exactly
			double sc = ldexp(1.0, e), isc = ldexp(1.0, -e);
			// origin two quanta below lo, rounded down to a float
			double want = (double)lo[a] - 2.0 * sc;
			float pf = (float)want;
			if ((double)pf > want)
				pf = nextafterf(pf, -FLT_MAX);
			double top = ((double)hi[a] - pf) * isc;
			if ((top + 2.0 <= 255.0 && e + kQExpBias >= 1) ||
			  e + kQExpBias >= 254) {
				p[a] = pf;
				ex[a] = e;
				break;
			}
		}
	}
	n->px = p[0];
	n->py = p[1];
	n->pz = p[2];
	n->ex = (uint8_t)(ex[0] + kQExpBias);
	n->ey = (uint8_t)(ex[1] + kQExpBias);
	n->ez = (uint8_t)(ex[2] + kQExpBias);
	uint8_t *qlo[3] = {n->qlox, n->qloy, n->qloz};
	uint8_t *qhi[3] = {n->qhix, n->qhiy, n->qhiz};
	for (int s = 0; s < 8; s++) {
		bool valid = cmin[s][0] <= cmax[s][0] &&
		  cmin[s][1] <= cmax[s][1] && cmin[s][2] <= cmax[s][2];
		for (int a = 0; a < 3; a++) {
			if (!valid) {
				qlo[a][s] = 255;
				qhi[a][s] = 0;
				continue;
			}
			double isc = ldexp(1.0, -ex[a]);
			double l = floor(((double)cmin[s][a] - p[a]) * isc -
			  kQMargin);
			double h = ceil(((double)cmax[s][a] - p[a]) * isc +
			  kQMargin);
			// both ends saturate: a child beyond the clamped frame
			// can lie wholly above 255 or below 0
			l = fmin(fmax(l, 0.0), 255.0);
			h = fmin(fmax(h, 0.0), 255.0);
			qlo[a][s] = (uint8_t)l;
			qhi[a][s] = (uint8_t)h;
		}
	}
}

} // namespace nb

#endif
