// Prints, for a cell count N given on the command line, whether the device
// layouts of the radiation fields R (6 N doubles) and the thermodynamics
// fields T (4 N doubles) map every (field, cell) pair to its own slot of the
// array, and whether the four optical depths of a cell fill one aligned
// 32-byte group and its two column densities one 16-byte pair.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "../../torch_b200/csrc/trg_types.h"

using namespace trg;

int main(int argc, char** argv) {
	const long long N = argc > 1 ? std::atoll(argv[1]) : 7;
	bool ok = true;
	std::vector<int> seen(6 * N, 0);
	for (int f = 0; f < NR; ++f)
		for (long long id = 0; id < N; ++id) {
			const long long k = r_index(N, f, id);
			if (k < 0 || k >= 6 * N || seen[k]++) ok = false;
		}
	for (long long id = 0; id < N; ++id) {
		const long long a = r_index(N, R_TAU, id);
		if (a % 4 != 0 || r_index(N, R_DTAU, id) != a + 1 || r_index(N, R_TAU_A, id) != a + 2 ||
		    r_index(N, R_DTAU_A, id) != a + 3)
			ok = false;
	}
	std::vector<int> seen_t(4 * N, 0);
	for (int f = 0; f < NT; ++f)
		for (long long id = 0; id < N; ++id) {
			const long long k = t_index(N, f, id);
			if (k < 0 || k >= 4 * N || seen_t[k]++) ok = false;
		}
	for (long long id = 0; id < N; ++id)
		if (t_index(N, T_COL_DEN, id) != 2 * id || t_index(N, T_DCOL_DEN, id) != 2 * id + 1) ok = false;
	std::printf("%s\n", ok ? "ok" : "bad");
	return ok ? 0 : 1;
}
