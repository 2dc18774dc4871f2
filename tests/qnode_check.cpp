// Checks of the node encoder shared by every tree build, host and device
// (nodebleed_b200/csrc/qnode.h), on random nodes that include extreme
// scales, infinite bounds, empty and NaN children.  Built and run by
// test_qnode_encoder.py; prints "ok <nodes>" or the first failure and exits
// non-zero.
//
// Per node: stored exponents within 1..254; a finite origin; every valid
// child whose bounds lie within the clamped frame (+-2^125) inside its
// planes with 1/32 of a quantum to spare, the planes rebuilt as the device
// does (origin + byte * 2^(exponent byte - 119)); invalid children (min >
// max, or NaN) as the empty slot 255 / 0.  Per slot assignment: every child
// a distinct slot, whatever the centres.

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <random>

#include "qnode.h"

namespace {

std::mt19937_64 rng(20261204);

double uni(double a, double b)
{
	return std::uniform_real_distribution<double>(a, b)(rng);
}

float coord(double scale)
{
	switch (rng() % 16) {
	case 0:
		return INFINITY;
	case 1:
		return -INFINITY;
	case 2:
		return FLT_MAX;
	case 3:
		return -FLT_MAX;
	default:
		return (float)(uni(-1.0, 1.0) * scale);
	}
}

int fail(const char *what, long node, int slot, int axis)
{
	std::printf("FAIL %s node %ld slot %d axis %d\n", what, node, slot,
	  axis);
	return 1;
}

} // namespace

int main(int argc, char **argv)
{
	long nodes = argc > 1 ? std::atol(argv[1]) : 200000;
	const double frame = std::ldexp(1.0, 125);
	for (long it = 0; it < nodes; it++) {
		float cmin[8][3], cmax[8][3];
		double scale = std::pow(10.0, uni(-38.0, 38.5));
		bool extreme = it % 4 == 0;
		for (int s = 0; s < 8; s++) {
			int kind = (int)(rng() % 8);
			for (int a = 0; a < 3; a++) {
				float x = extreme ? coord(scale) :
				  (float)(uni(-1.0, 1.0) * scale);
				float y = extreme ? coord(scale) :
				  (float)(uni(-1.0, 1.0) * scale);
				cmin[s][a] = std::fmin(x, y);
				cmax[s][a] = std::fmax(x, y);
			}
			if (kind == 0) { // empty
				cmin[s][0] = 1.0f;
				cmax[s][0] = -1.0f;
			} else if (kind == 1 && extreme) {
				cmin[s][rng() % 3] = NAN;
			}
		}
		nb_qnode q;
		nb::quantise_node_hd(cmin, cmax, &q);
		const float p[3] = {q.px, q.py, q.pz};
		const uint8_t e[3] = {q.ex, q.ey, q.ez};
		const uint8_t *lo[3] = {q.qlox, q.qloy, q.qloz};
		const uint8_t *hi[3] = {q.qhix, q.qhiy, q.qhiz};
		for (int a = 0; a < 3; a++) {
			if (e[a] < 1 || e[a] > 254)
				return fail("exponent", it, -1, a);
			if (!std::isfinite(p[a]))
				return fail("origin", it, -1, a);
		}
		for (int s = 0; s < 8; s++) {
			bool valid = cmin[s][0] <= cmax[s][0] &&
			  cmin[s][1] <= cmax[s][1] && cmin[s][2] <= cmax[s][2];
			for (int a = 0; a < 3; a++) {
				if (!valid) {
					if (lo[a][s] != 255 || hi[a][s] != 0)
						return fail("empty slot", it, s, a);
					continue;
				}
				if (!(cmin[s][a] >= -frame && cmax[s][a] <= frame))
					continue;
				double sc = std::ldexp(1.0, (int)e[a] - nb::kQExpBias);
				double ql = (double)p[a] + lo[a][s] * sc;
				double qh = (double)p[a] + hi[a][s] * sc;
				if (!(ql <= (double)cmin[s][a] - sc / 32.0))
					return fail("low plane", it, s, a);
				if (!(qh >= (double)cmax[s][a] + sc / 32.0))
					return fail("high plane", it, s, a);
			}
		}
		// slot assignment on the same node's centres (overflowing to inf
		// and NaN in the extreme nodes) against a random node centre
		int n = 1 + (int)(rng() % 8);
		float cen[8][3], nc[3];
		for (int c = 0; c < n; c++)
			for (int a = 0; a < 3; a++)
				cen[c][a] = 0.5f * (cmin[c][a] + cmax[c][a]);
		for (int a = 0; a < 3; a++)
			nc[a] = extreme ? coord(scale) : (float)uni(-scale, scale);
		int slot_of[8];
		nb::assign_slots(n, cen, nc, slot_of);
		unsigned used = 0;
		for (int c = 0; c < n; c++) {
			if (slot_of[c] < 0 || slot_of[c] > 7 ||
			  (used >> slot_of[c] & 1u))
				return fail("slot", it, c, -1);
			used |= 1u << slot_of[c];
		}
	}
	std::printf("ok %ld\n", nodes);
	return 0;
}
