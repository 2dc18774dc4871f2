// The warp form of the greedy slot assignment (tc_assign_slots_warp in
// nodebleed_b200/csrc/tlas_cta.cuh) restated on the CPU with 32 emulated
// lanes, against the sequential assign_slots of qnode.h that the other
// builds use: each lane scores pairs lane and lane + 32 (child = pair / 8,
// slot = pair % 8), scores clamped to -FLT_MAX; each round a butterfly
// argmax over xor distances 16..1, the lower pair index winning equal
// scores.  Random nodes, a quarter with NaN / +-inf / +-FLT_MAX centres.
// Built and run by test_qnode_encoder.py; prints "ok <nodes>" or the first
// difference and exits non-zero.

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "qnode.h"

namespace {

// returns false when the lanes' winners disagree
bool warp_assign(int nchild, const float cen[8][3], const float nc[3],
                 int slot_of[8])
{
	float sc[32][2];
	bool ok[32][2];
	for (int lane = 0; lane < 32; lane++)
		for (int h = 0; h < 2; h++) {
			int p = lane + 32 * h, c = p >> 3, sl = p & 7;
			ok[lane][h] = c < nchild;
			float v = 0.0f;
			if (ok[lane][h])
				for (int a = 0; a < 3; a++)
					v += (cen[c][a] - nc[a]) *
					  ((sl >> a) & 1 ? 1.0f : -1.0f);
			sc[lane][h] = std::fmax(v, -FLT_MAX);
		}
	for (int i = 0; i < 8; i++)
		slot_of[i] = -1;
	for (int r = 0; r < nchild; r++) {
		float bv[32];
		int bi[32];
		for (int lane = 0; lane < 32; lane++) {
			bv[lane] = -FLT_MAX;
			bi[lane] = -1;
			for (int h = 0; h < 2; h++)
				if (ok[lane][h] &&
				  (bi[lane] < 0 || sc[lane][h] > bv[lane])) {
					bv[lane] = sc[lane][h];
					bi[lane] = lane + 32 * h;
				}
		}
		for (int o = 16; o > 0; o >>= 1) {
			float nv[32];
			int ni[32];
			for (int lane = 0; lane < 32; lane++) {
				float ov = bv[lane ^ o];
				int oi = bi[lane ^ o];
				nv[lane] = bv[lane];
				ni[lane] = bi[lane];
				if (oi >= 0 && (bi[lane] < 0 || ov > bv[lane] ||
				  (ov == bv[lane] && oi < bi[lane]))) {
					nv[lane] = ov;
					ni[lane] = oi;
				}
			}
			for (int lane = 0; lane < 32; lane++) {
				bv[lane] = nv[lane];
				bi[lane] = ni[lane];
			}
		}
		for (int lane = 1; lane < 32; lane++)
			if (bi[lane] != bi[0])
				return false;
		if (bi[0] < 0)
			return false;
		int bc = bi[0] >> 3, bs = bi[0] & 7;
		slot_of[bc] = bs;
		for (int lane = 0; lane < 32; lane++)
			for (int h = 0; h < 2; h++) {
				int p = lane + 32 * h;
				if ((p >> 3) == bc || (p & 7) == bs)
					ok[lane][h] = false;
			}
	}
	return true;
}

} // namespace

int main(int argc, char **argv)
{
	long nodes = argc > 1 ? std::atol(argv[1]) : 1000000;
	std::mt19937 g(9);
	std::uniform_real_distribution<float> U(-3.0f, 3.0f);
	const float odd[5] = {INFINITY, -INFINITY, NAN, FLT_MAX, -FLT_MAX};
	for (long it = 0; it < nodes; it++) {
		int n = 1 + (int)(g() % 8);
		float cen[8][3], nc[3];
		for (int a = 0; a < 3; a++)
			nc[a] = U(g);
		// repeated coordinates make equal scores, the tie-break's case
		for (int c = 0; c < n; c++)
			for (int a = 0; a < 3; a++)
				cen[c][a] = g() % 3 == 0 ? nc[a] :
				  (g() % 5 == 0 && c > 0 ? cen[0][a] : U(g));
		if (it % 4 == 1)
			for (int c = 0; c < n; c++)
				for (int a = 0; a < 3; a++) {
					unsigned k = g() % 9;
					if (k < 5)
						cen[c][a] = odd[k];
				}
		if (it % 8 == 3)
			nc[g() % 3] = g() & 1 ? INFINITY : NAN;
		int s1[8], s2[8];
		nb::assign_slots(n, cen, nc, s1);
		if (!warp_assign(n, cen, nc, s2)) {
			std::printf("FAIL lanes disagree at node %ld\n", it);
			return 1;
		}
		for (int c = 0; c < n; c++)
			if (s1[c] != s2[c] || s1[c] < 0) {
				std::printf("FAIL node %ld child %d: %d vs %d\n", it,
				  c, s1[c], s2[c]);
				return 1;
			}
	}
	std::printf("ok %ld\n", nodes);
	return 0;
}
