// Taylor-Green vortex with the cumulant collision (Geier 2017 + anti-aliasing),
// the configuration of TNL-LBM's sim_NSE/sim_4.cu, through the C++ interface.
//
//   sim_tgv [N] [steps] [probe_period] [storage: f64|f32|f16s|bf16s]
//
// Prints "iteration kinetic_energy enstrophy" in lattice units on even
// iterations (sim_4.cu:369-372 probes even iterations only); KE and
// enstrophy follow sim_4.cu:257-301.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "lbm_b200.hpp"

using namespace tnl_lbm_b200;

template <class STORAGE>
int run(int N, int steps, int period)
{
	using CONFIG = LBM_CONFIG<STORAGE, D3Q27_CUM<CUM_2017_ANTIALIAS>, D3Q27_EQ_INV_CUM>;
	const double u0 = 0.05, Re = 1600.0;
	const double nu = u0 * (N / (2 * M_PI)) / Re;
	Lattice<CONFIG> lat(N, N, N, nu, /*periodic=*/true);
	lat.init_taylor_green(u0);
	std::printf("# N=%d nu=%.6e u0=%g Re=%g\n# iter kinetic_energy enstrophy\n", N, nu, u0, Re);
	for (int it = 0; it < steps; it += period) {
		const int n = it + period <= steps ? period : steps - it;
		lat.step(n, LBM_STEP_SUMS | LBM_STEP_MACRO);
		const Sums s = lat.sums();
		const double V = (double) N * N * N;
		std::printf("%lld %.12e %.12e\n", (long long) lat.iteration(), s.kinetic_energy(1.0, lat.sites()),
					lat.enstrophy_sum() / 2.0 / V);
	}
	return 0;
}

int main(int argc, char** argv)
{
	const int N = argc > 1 ? std::atoi(argv[1]) : 64;
	const int steps = argc > 2 ? std::atoi(argv[2]) : 1000;
	int period = argc > 3 ? std::atoi(argv[3]) : 10;
	const char* st = argc > 4 ? argv[4] : "f32";
	if (period % 2)
		period++;
	try {
		if (!std::strcmp(st, "f64"))
			return run<F64>(N, steps, period);
		if (!std::strcmp(st, "f16s"))
			return run<F16S>(N, steps, period);
		if (!std::strcmp(st, "bf16s"))
			return run<BF16S>(N, steps, period);
		return run<F32>(N, steps, period);
	}
	catch (const Error& e) {
		std::fprintf(stderr, "error %d: %s\n", e.code(), e.what());
		return 2;
	}
}
