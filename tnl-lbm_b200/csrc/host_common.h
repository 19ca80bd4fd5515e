// Host-side helpers shared by the single-lattice and the ensemble C-ABI:
// population layout of one lattice and the per-viscosity collision constants.
#pragma once

#include "launch.h"

namespace lbm {

// Storage layout of one X x Y x Z lattice with its ghost layer, for elements
// of es bytes: rows start 128-byte aligned at interior x = 0 (x0 elements of
// front pad, ghost x = -1 at x0 - 1); a row holds the X interior sites, the
// ghost x = X and room for the tile kernel's odd-step window, which reaches up
// to 2 x 16 bytes beyond the last site.  f is left null.
inline Geometry make_geometry(int X, int Y, int Z, int es, int slots = 27)
{
	// Rows of `row` elements (interior from x0, 128-byte aligned, with room for
	// 16-byte windows past both ends).  The `slots` rows of one (y, z) lattice
	// row lie side by side (slot q at q * sq within the group), so the 27
	// streams a warp reads for one row of sites sit in one contiguous region of
	// 27 rows instead of 27 planes a lattice-size apart: about 3 % more HBM
	// throughput for the step kernels than separate planes per slot.
	Geometry g{};
	const int align = 128 / es;	 // elements per 128 bytes
	const int a16 = 16 / es;
	const int row = ((align + X + 2 * a16 + align - 1) / align) * align;
	g.x0 = align;
	g.sq = row;
	g.sy = slots * row;
	g.sz = g.sy * (Y + 2);
	g.X = X;
	g.Y = Y;
	g.Z = Z;
	return g;
}

// elements of the allocation of a geometry (all slots, ghost layer included)
inline size_t geometry_elems(const Geometry& g)
{
	return (size_t) g.sz * (size_t) (g.Z + 2);
}

// Geier 2017 relaxation rates for omega2 = 1 (col_cum.h:195-228), evaluated
// once per viscosity in double precision
inline void cumulant_rates(double nu, CollParamsD& p)
{
	const double w1 = 1.0 / (3.0 * nu + 0.5);
	const double w2 = 1.0;
	p.w1 = w1;
	p.w3 = 8 * (w1 - 2) * (w2 * (3 * w1 - 1) - 5 * w1) / (8 * (5 - 2 * w1) * w1 + w2 * (8 + w1 * (9 * w1 - 26)));
	p.w4 = 8 * (w1 - 2) * (w1 + w2 * (3 * w1 - 7)) / (w2 * (56 - 42 * w1 + 9 * w1 * w1) - 8 * w1);
	p.w5 = 24 * (w1 - 2) * (4 * w1 * w1 + w1 * w2 * (18 - 13 * w1) + w2 * w2 * (2 + w1 * (6 * w1 - 11)))
		 / (16 * w1 * w1 * (w1 - 6) - 2 * w1 * w2 * (216 + 5 * w1 * (9 * w1 - 46))
			+ w2 * w2 * (w1 * (3 * w1 - 10) * (15 * w1 - 28) - 48));
	p.A = (4 * w1 * w1 + 2 * w1 * w2 * (w1 - 6) + w2 * w2 * (w1 * (10 - 3 * w1) - 4)) / (w1 - w2) / (w2 * (2 + 3 * w1) - 8 * w1);
	p.B = (4 * w1 * w2 * (9 * w1 - 16) - 4 * w1 * w1 - 2 * w2 * w2 * (2 + 9 * w1 * (w1 - 2))) / 3.0 / (w1 - w2)
		/ (w2 * (2 + 3 * w1) - 8 * w1);
	p.tau = 3.0 * nu + 0.5;
}

}  // namespace lbm
