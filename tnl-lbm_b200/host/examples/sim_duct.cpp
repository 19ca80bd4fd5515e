// Rectangular duct with a velocity inlet and a fixed-density outlet, the
// configuration of TNL-LBM's sim_NSE/sim_2.cu in velocity-inlet mode: walls
// one site inside GEO_NOTHING rims (sim_2.cu:140-157), default cumulant.
//
//   sim_duct [X] [Y] [Z] [steps] [u_max] [Re]
//
// Prints the mass, the mean streamwise velocity and the kinetic energy every
// steps/10 iterations.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "lbm_b200.hpp"

using namespace tnl_lbm_b200;

int main(int argc, char** argv)
{
	const int X = argc > 1 ? std::atoi(argv[1]) : 256;
	const int Y = argc > 2 ? std::atoi(argv[2]) : 64;
	const int Z = argc > 3 ? std::atoi(argv[3]) : 64;
	const int steps = argc > 4 ? std::atoi(argv[4]) : 2000;
	const double u_max = argc > 5 ? std::atof(argv[5]) : 0.04;
	const double Re = argc > 6 ? std::atof(argv[6]) : 2000.0;
	const double H = Y - 2.0;  // distance between the wall nodes
	const double nu = u_max * H / Re;
	using CONFIG = LBM_CONFIG<F32, D3Q27_CUM<CUM_DEFAULT>, D3Q27_EQ_INV_CUM>;
	try {
		Lattice<CONFIG> lat(X, Y, Z, nu);
		std::vector<uint8_t> map((size_t) X * Y * Z, GEO_FLUID);
		auto at = [&](int x, int y, int z) -> uint8_t& { return map[((size_t) z * Y + y) * X + x]; };
		for (int z = 0; z < Z; z++)
			for (int y = 0; y < Y; y++)
				for (int x = 0; x < X; x++) {
					uint8_t g = GEO_FLUID;
					if (x == 0)
						g = GEO_INFLOW_LEFT;
					if (x == X - 1)
						g = GEO_OUTFLOW_EQ;
					if (y == 1 || y == Y - 2 || z == 1 || z == Z - 2)
						g = GEO_WALL;
					if (y == 0 || y == Y - 1 || z == 0 || z == Z - 1)
						g = GEO_NOTHING;
					at(x, y, z) = g;
				}
		lat.set_map(map);
		std::vector<double> prof((size_t) Y * Z, 0.0);
		for (int z = 2; z < Z - 2; z++)
			for (int y = 2; y < Y - 2; y++) {
				const double a = (y - 1.0) / (Y - 3.0), b = (z - 1.0) / (Z - 3.0);
				prof[(size_t) z * Y + y] = u_max * 16 * a * (1 - a) * b * (1 - b);
			}
		lat.set_inflow(prof);
		lat.init_equilibrium();
		std::printf("# duct %dx%dx%d nu=%.6e u_max=%g Re=%g\n# iter mass mean_ux kinetic_energy\n", X, Y, Z, nu, u_max, Re);
		const int period = steps >= 10 ? steps / 10 : 1;
		for (int it = 0; it < steps; it += period) {
			lat.step(period, LBM_STEP_SUMS);
			const Sums s = lat.sums();
			std::printf("%lld %.10e %.10e %.10e\n", (long long) lat.iteration(), s.mass, s.momentum[0] / s.mass,
						s.kinetic_energy(1.0, lat.sites()));
		}
	}
	catch (const Error& e) {
		std::fprintf(stderr, "error %d: %s\n", e.code(), e.what());
		return 2;
	}
	return 0;
}
