// Oracle-only stand-in for the TNL header that TNL-LBM's per-site operator
// headers include (include/lbm3d/d3q27/eq.h:3, eq_inv_cum.h:3, macro.h:5).
// It supplies only what those headers use on the host: the
// `__cuda_callable__` qualifier and the TNL::Backend::ldg / TNL::swap helpers
// (streaming_AA.h:84, bc.h:208).  Test infrastructure: never linked into the
// product library.
#pragma once

#include <algorithm>
#include <cmath>
#include <utility>

#ifndef __cuda_callable__
	#define __cuda_callable__
#endif

namespace TNL {
namespace Backend {
template <typename T>
inline T ldg(const T& value)
{
	return value;
}
}  // namespace Backend

template <typename T>
inline void swap(T& a, T& b)
{
	T tmp = a;
	a = b;
	b = tmp;
}

template <typename T>
inline T min(const T& a, const T& b)
{
	return a < b ? a : b;
}

template <typename T>
inline T max(const T& a, const T& b)
{
	return a > b ? a : b;
}
}  // namespace TNL
