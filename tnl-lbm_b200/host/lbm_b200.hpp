// C++ host interface of the B200 D3Q27 A-A hot path.
//
// Mirrors the compile-time composition of TNL-LBM (LBM_CONFIG,
// include/lbm3d/defs.h:288-310) with tag types for the storage format, the
// collision slot (COLL) and the equilibrium (EQ), and wraps one lattice of the
// C-ABI (include/tnl_lbm_b200.h) in a move-only RAII class.  Errors throw
// tnl_lbm_b200::Error with the library's status code and message.
//
//     using CONFIG = tnl_lbm_b200::LBM_CONFIG<tnl_lbm_b200::F32,
//                                             tnl_lbm_b200::D3Q27_CUM<tnl_lbm_b200::CUM_2017_ANTIALIAS>,
//                                             tnl_lbm_b200::D3Q27_EQ_INV_CUM>;
//     tnl_lbm_b200::Lattice<CONFIG> lat(64, 64, 64, nu, /*periodic=*/true);
//     lat.init_taylor_green(0.05);
//     lat.step(1000, LBM_STEP_SUMS);
//     auto s = lat.sums();
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "tnl_lbm_b200.h"

namespace tnl_lbm_b200 {

// ---- storage formats (the TRAITS::dreal choice plus the shifted formats)
struct F64
{
	static constexpr int id = LBM_STORE_F64;
};
struct F32
{
	static constexpr int id = LBM_STORE_F32;
};
struct F32S
{
	static constexpr int id = LBM_STORE_F32S;
};
struct F16S
{
	static constexpr int id = LBM_STORE_F16S;
};
struct BF16S
{
	static constexpr int id = LBM_STORE_BF16S;
};

// ---- collision slot (D3Q27_CUM, D3Q27_SRT, D3Q27_BGK, D3Q27_MRT)
constexpr int CUM_DEFAULT = 0;
constexpr int CUM_ANTIALIAS = LBM_CUM_ANTIALIAS;
constexpr int CUM_2017_ANTIALIAS = LBM_CUM_GEIER_2017 | LBM_CUM_ANTIALIAS;

template <int FLAGS = CUM_DEFAULT>
struct D3Q27_CUM
{
	static constexpr int id = LBM_COLL_CUM;
	static constexpr int flags = FLAGS;
	static constexpr const char* name = "CUM";
};
struct D3Q27_SRT
{
	static constexpr int id = LBM_COLL_SRT;
	static constexpr int flags = 0;
	static constexpr const char* name = "SRT";
};
struct D3Q27_BGK
{
	static constexpr int id = LBM_COLL_BGK;
	static constexpr int flags = 0;
	static constexpr const char* name = "BGK";
};
struct D3Q27_MRT
{
	static constexpr int id = LBM_COLL_MRT;
	static constexpr int flags = 0;
	static constexpr const char* name = "MRT_LES";
};

// ---- equilibrium (D3Q27_EQ, D3Q27_EQ_INV_CUM)
struct D3Q27_EQ
{
	static constexpr int id = LBM_EQ_SECOND_ORDER;
};
struct D3Q27_EQ_INV_CUM
{
	static constexpr int id = LBM_EQ_INV_CUM;
};

template <class STORAGE, class COLL, class EQ>
struct LBM_CONFIG
{
	using storage = STORAGE;
	using coll = COLL;
	using eq = EQ;
};

// GEO site types of D3Q27_BC_All (include/lbm3d/d3q27/bc.h:17-43)
enum GEO : uint8_t
{
	GEO_FLUID = 0,
	GEO_WALL = 1,
	GEO_INFLOW = 2,
	GEO_INFLOW_LEFT = 3,
	GEO_INFLOW_BB_LEFT = 4,
	GEO_INFLOW_EQ_LEFT = 5,
	GEO_OUTFLOW_EQ = 6,
	GEO_OUTFLOW_RIGHT = 7,
	GEO_OUTFLOW_RIGHT_INTERP = 8,
	GEO_PERIODIC = 9,
	GEO_NOTHING = 10,
	GEO_SYM_TOP = 11,
	GEO_SYM_BOTTOM = 12,
	GEO_SYM_LEFT = 13,
	GEO_SYM_RIGHT = 14,
	GEO_SYM_BACK = 15,
	GEO_SYM_FRONT = 16,
};

class Error : public std::runtime_error
{
public:
	Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
	int code() const
	{
		return code_;
	}

private:
	int code_;
};

inline void check(int rc)
{
	if (rc != LBM_OK)
		throw Error(rc, lbm_last_error());
}

// sums of one observed step (lbm_get_sums)
struct Sums
{
	double mass = 0, momentum[3] = {0, 0, 0}, rho_u2 = 0, nonfinite = 0;
	// kinetic energy sum rho |u|^2 / (2 rho0 V) of sim_NSE/sim_4.cu:257-275
	double kinetic_energy(double rho0, long long volume) const
	{
		return rho_u2 / rho0 / 2.0 / (double) volume;
	}
};

template <class CONFIG>
class Lattice
{
public:
	Lattice(int X, int Y, int Z, double viscosity, bool periodic = false, double fx = 0, double fy = 0, double fz = 0,
			int device = 0, bool use_graphs = true)
		: X_(X), Y_(Y), Z_(Z)
	{
		lbm_desc d{};
		d.X = X;
		d.Y = Y;
		d.Z = Z;
		d.storage = CONFIG::storage::id;
		d.collision = CONFIG::coll::id;
		d.cum_flags = CONFIG::coll::flags;
		d.equilibrium = CONFIG::eq::id;
		d.periodic = periodic ? 1 : 0;
		d.viscosity = viscosity;
		d.fx = fx;
		d.fy = fy;
		d.fz = fz;
		d.device = device;
		d.use_graphs = use_graphs ? 1 : 0;
		check(lbm_create(&d, &h_));
	}
	~Lattice()
	{
		if (h_)
			lbm_destroy(h_);
	}
	Lattice(const Lattice&) = delete;
	Lattice& operator=(const Lattice&) = delete;
	Lattice(Lattice&& o) noexcept : h_(std::exchange(o.h_, nullptr)), X_(o.X_), Y_(o.Y_), Z_(o.Z_) {}

	long long sites() const
	{
		return (long long) X_ * Y_ * Z_;
	}
	lbm_handle handle() const
	{
		return h_;
	}

	void set_map(const std::vector<uint8_t>& map)
	{
		if ((long long) map.size() != sites())
			throw Error(LBM_ERR_INVALID, "map size does not match the lattice");
		check(lbm_set_map(h_, map.data()));
	}
	void set_inflow(const std::vector<double>& vx, const std::vector<double>& vy = {}, const std::vector<double>& vz = {})
	{
		check(lbm_set_inflow(h_, vx.empty() ? nullptr : vx.data(), vy.empty() ? nullptr : vy.data(),
							 vz.empty() ? nullptr : vz.data()));
	}
	void set_viscosity(double nu)
	{
		check(lbm_set_viscosity(h_, nu));
	}
	void init_equilibrium(double rho0 = 1, double vx0 = 0, double vy0 = 0, double vz0 = 0)
	{
		check(lbm_init_equilibrium(h_, nullptr, nullptr, nullptr, nullptr, rho0, vx0, vy0, vz0));
	}
	void init_equilibrium(const std::vector<double>& rho, const std::vector<double>& vx, const std::vector<double>& vy,
						  const std::vector<double>& vz)
	{
		check(lbm_init_equilibrium(h_, rho.data(), vx.data(), vy.data(), vz.data(), 1, 0, 0, 0));
	}
	void init_taylor_green(double u0, double rho0 = 1)
	{
		check(lbm_init_taylor_green(h_, u0, rho0));
	}
	void step(int64_t n, int flags = 0)
	{
		check(lbm_step(h_, n, flags));
	}
	int64_t iteration() const
	{
		return lbm_iteration(h_);
	}
	Sums sums() const
	{
		double s[6];
		check(lbm_get_sums(h_, s));
		Sums r;
		r.mass = s[0];
		r.momentum[0] = s[1];
		r.momentum[1] = s[2];
		r.momentum[2] = s[3];
		r.rho_u2 = s[4];
		r.nonfinite = s[5];
		return r;
	}
	std::vector<double> macro() const
	{
		std::vector<double> m(4 * (size_t) sites());
		check(lbm_get_macro(h_, m.data()));
		return m;
	}
	double enstrophy_sum() const
	{
		double e = 0;
		check(lbm_enstrophy_sum(h_, &e));
		return e;
	}
	std::vector<double> populations(int layout = LBM_LAYOUT_GHOST) const
	{
		const int g = layout == LBM_LAYOUT_GHOST ? 2 : 0;
		std::vector<double> f(27 * (size_t) (X_ + g) * (Y_ + g) * (Z_ + g));
		check(lbm_get_populations(h_, f.data(), layout, LBM_DTYPE_F64));
		return f;
	}
	void set_populations(const std::vector<double>& f, int layout = LBM_LAYOUT_GHOST)
	{
		check(lbm_set_populations(h_, f.data(), layout, LBM_DTYPE_F64));
	}
	void autotune(int ntrials = 4)
	{
		check(lbm_autotune(h_, ntrials));
	}
	void synchronize() const
	{
		check(lbm_synchronize(h_));
	}

private:
	lbm_handle h_ = nullptr;
	int X_, Y_, Z_;
};

}  // namespace tnl_lbm_b200
