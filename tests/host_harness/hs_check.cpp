// Test harness (CPU only): exposes the library's host-side set-up, which runs
// before any CUDA call, so that CPU tests can check parameter validation and
// the sweep order without a GPU.
#include <cstring>
#include <string>

#include "../../torch_b200/csrc/setup.h"

extern "C" int hs_check(const trg_params* p, const double* den, const double* pre, const double* hii,
                        const double* v0, const double* v1, const double* v2, char* err, int errlen,
                        long long* nshell_all, long long* nshell_nonwind, long long* first_nonwind,
                        long long* nwind) {
	trg::HostSetup hs;
	std::string why = trg::host_setup(*p, den, pre, hii, v0, v1, v2, nullptr, hs);
	if (!why.empty()) {
		std::strncpy(err, why.c_str(), errlen - 1);
		err[errlen - 1] = 0;
		return 1;
	}
	*nshell_all = (long long)hs.off_all.size() - 1;
	*nshell_nonwind = (long long)hs.off_nonwind.size() - 1;
	*first_nonwind = hs.first_nonwind_cell;
	*nwind = (long long)hs.wind_cells.size();
	return 0;
}
