/*
 * ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * A C-callable driver around the UNMODIFIED ALP reference backends.  It is
 * compiled by oracle/Makefile against the reference's own headers and
 * sources (never copied here), once with -D_GRB_BACKEND=reference and once
 * with -D_GRB_BACKEND=reference_omp, into the git-ignored oracle/_ref/.
 * Its uses:
 *   - pin the C restatement (alp_oracle.c) to the reference's behaviour;
 *   - golden vectors for the GPU parity tests (tests/golden/make_golden.py);
 *   - the timed CPU baseline of bench.py (reference_omp on the host cores).
 *
 * Every entry point builds the ALP containers from plain arrays through the
 * public API (grb::buildMatrixUnique, grb::setElement), runs the public
 * primitive or algorithm, and exports the result.  Times are wall-clock ms
 * of the primitive/algorithm call alone (container build excluded).
 */
#include <graphblas.hpp>
#include <graphblas/algorithms/conjugate_gradient.hpp>
#include <graphblas/algorithms/simple_pagerank.hpp>
#include <graphblas/algorithms/hpcg/hpcg.hpp>
#include <graphblas/algorithms/hpcg/system_building_utils.hpp>

#include <array>
#include <chrono>
#include <memory>
#include <cstdint>
#include <cstring>
#include <vector>

using namespace grb;

namespace {

enum { T_VOID = 0, T_BOOL = 1, T_INT32 = 2, T_FP64 = 3 };
enum {
	R_PT_F64 = 0, R_LORLAND = 1, R_MINPLUS_I32 = 2, R_PATTERN_F64 = 3, R_PT_I32 = 4,
	R_PLUS_RIGHTIF_U64 = 5, R_MAX_LEFTIF_U64 = 6, R_TIMES_PLUS_F64 = 7
};

bool g_init = false;
void ensure_init() {
	if (!g_init) {
		grb::init();
		g_init = true;
	}
}

double now_ms() {
	return std::chrono::duration<double, std::milli>(
		std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename D>
RC build_matrix(Matrix<D> &A, int64_t nnz, const uint32_t *I, const uint32_t *J, const void *V,
	IOMode mode) {
	std::vector<size_t> Ii(I, I + nnz), Jj(J, J + nnz);
	const D *vals = static_cast<const D *>(V);
	return buildMatrixUnique(A, Ii.data(), Jj.data(), vals, size_t(nnz), mode);
}

// a vector with entries only where assigned (all if assigned == nullptr)
template <typename D>
RC build_vector(Vector<D> &x, int64_t n, const void *vals, const uint8_t *assigned) {
	RC rc = clear(x);
	const D *v = static_cast<const D *>(vals);
	for (int64_t i = 0; rc == SUCCESS && i < n; ++i)
		if (!assigned || assigned[i]) rc = setElement(x, v[i], size_t(i));
	return rc;
}

template <typename D>
void export_vector(const Vector<D> &x, int64_t n, void *vals, uint8_t *assigned) {
	D *v = static_cast<D *>(vals);
	if (assigned) std::memset(assigned, 0, size_t(n));
	for (const auto &p : x) {
		v[p.first] = p.second;
		if (assigned) assigned[p.first] = 1;
	}
}

// ------------------------------------------------------------------ mxv --
template <Descriptor descr, typename D, class Ring>
RC run_mxv(int vxm_form, Vector<D> &u, const Vector<bool> &um, const Matrix<D> &A,
	const Vector<D> &v, const Vector<bool> &vm, const Ring &ring) {
	if (vxm_form) return vxm<descr>(u, um, v, vm, A, ring);
	return mxv<descr>(u, um, A, v, vm, ring);
}

template <typename D, class Ring>
RC mxv_descr(uint32_t descr, int vxm_form, Vector<D> &u, const Vector<bool> &um,
	const Matrix<D> &A, const Vector<D> &v, const Vector<bool> &vm, const Ring &ring) {
	using namespace descriptors;
	switch (descr) {
	case no_operation: return run_mxv<no_operation>(vxm_form, u, um, A, v, vm, ring);
#ifdef ALPO_FULL_SET
	case invert_mask: return run_mxv<invert_mask>(vxm_form, u, um, A, v, vm, ring);
	case structural: return run_mxv<structural>(vxm_form, u, um, A, v, vm, ring);
	case structural | invert_mask:
		return run_mxv<structural | invert_mask>(vxm_form, u, um, A, v, vm, ring);
	case add_identity: return run_mxv<add_identity>(vxm_form, u, um, A, v, vm, ring);
	case use_index: return run_mxv<use_index>(vxm_form, u, um, A, v, vm, ring);
	case explicit_zero: return run_mxv<explicit_zero>(vxm_form, u, um, A, v, vm, ring);
	case transpose_matrix: return run_mxv<transpose_matrix>(vxm_form, u, um, A, v, vm, ring);
#endif
	case dense: return run_mxv<dense>(vxm_form, u, um, A, v, vm, ring);
	}
	return UNSUPPORTED;
}

template <typename D, class Ring>
int mxv_ring(const Ring &ring, uint32_t descr, int vxm_form, int64_t m, int64_t n, int64_t nnz,
	const uint32_t *I, const uint32_t *J, const void *V, void *u, uint8_t *u_assigned,
	const uint8_t *u_mask, const uint8_t *u_mask_assigned, int has_u_mask, const void *v,
	const uint8_t *v_assigned, const uint8_t *v_mask, const uint8_t *v_mask_assigned,
	int has_v_mask, int reps, double *ms) {
	Matrix<D> A(static_cast<size_t>(m), static_cast<size_t>(n), static_cast<size_t>(nnz));
	RC rc = build_matrix<D>(A, nnz, I, J, V, SEQUENTIAL);
	const int64_t ulen = vxm_form ? n : m, vlen = vxm_form ? m : n;
	const bool tr = (descr & descriptors::transpose_matrix) != 0;
	const int64_t uo = tr ? vlen : ulen, vo = tr ? ulen : vlen;
	Vector<D> uu(static_cast<size_t>(uo)), vv(static_cast<size_t>(vo));
	Vector<bool> um(has_u_mask ? static_cast<size_t>(uo) : 0), vm(has_v_mask ? static_cast<size_t>(vo) : 0);
	if (rc == SUCCESS) rc = build_vector<D>(vv, vo, v, v_assigned);
	if (rc == SUCCESS && has_u_mask) rc = build_vector<bool>(um, uo, u_mask, u_mask_assigned);
	if (rc == SUCCESS && has_v_mask) rc = build_vector<bool>(vm, vo, v_mask, v_mask_assigned);
	if (rc != SUCCESS) return int(rc);
	double total = 0;
	for (int r = 0; r < (reps > 0 ? reps : 1); ++r) {
		rc = build_vector<D>(uu, uo, u, u_assigned);
		if (rc != SUCCESS) return int(rc);
		const double t0 = now_ms();
		rc = mxv_descr<D>(descr, vxm_form, uu, um, A, vv, vm, ring);
		total += now_ms() - t0;
		if (rc != SUCCESS) return int(rc);
	}
	if (ms) *ms = total / (reps > 0 ? reps : 1);
	export_vector<D>(uu, uo, u, u_assigned);
	return int(rc);
}

} // namespace

extern "C" {

__attribute__((visibility("default"))) int refw_threads(void) {
#ifdef _GRB_WITH_OMP
	return omp_get_max_threads();
#else
	return 1;
#endif
}

/* u (+)= A (x) v (vxm_form = 0) or v (x) A (vxm_form = 1) through grb::mxv /
 * grb::vxm with the given descriptor (one of the instantiated set), output
 * and input masks (Vector<bool>, has_*_mask = 0 for none), matrix from
 * (I, J, V) triples of the ring's type; u, v as value + assigned arrays. */
__attribute__((visibility("default"))) int refw_mxv(int ring, uint32_t descr, int vxm_form,
	int64_t m, int64_t n, int64_t nnz, const uint32_t *I, const uint32_t *J, const void *V,
	void *u, uint8_t *u_assigned, const uint8_t *u_mask, const uint8_t *u_mask_assigned,
	int has_u_mask, const void *v, const uint8_t *v_assigned, const uint8_t *v_mask,
	const uint8_t *v_mask_assigned, int has_v_mask, int reps, double *ms) {
	ensure_init();
	switch (ring) {
	case R_PT_F64: {
		Semiring<operators::add<double>, operators::mul<double>, identities::zero, identities::one> r;
		return mxv_ring<double>(r, descr, vxm_form, m, n, nnz, I, J, V, u, u_assigned, u_mask,
			u_mask_assigned, has_u_mask, v, v_assigned, v_mask, v_mask_assigned, has_v_mask, reps, ms);
	}
	case R_LORLAND: {
		Semiring<operators::logical_or<bool>, operators::logical_and<bool>,
			identities::logical_false, identities::logical_true> r;
		return mxv_ring<bool>(r, descr, vxm_form, m, n, nnz, I, J, V, u, u_assigned, u_mask,
			u_mask_assigned, has_u_mask, v, v_assigned, v_mask, v_mask_assigned, has_v_mask, reps, ms);
	}
	case R_MINPLUS_I32: {
		Semiring<operators::min<int>, operators::add<int>, identities::infinity, identities::zero> r;
		return mxv_ring<int>(r, descr, vxm_form, m, n, nnz, I, J, V, u, u_assigned, u_mask,
			u_mask_assigned, has_u_mask, v, v_assigned, v_mask, v_mask_assigned, has_v_mask, reps, ms);
	}
#ifdef ALPO_FULL_SET
	case R_PATTERN_F64: {
		Semiring<operators::add<double>, operators::left_assign_if<double, bool, double>,
			identities::zero, identities::logical_true> r;
		return mxv_ring<double>(r, descr, vxm_form, m, n, nnz, I, J, V, u, u_assigned, u_mask,
			u_mask_assigned, has_u_mask, v, v_assigned, v_mask, v_mask_assigned, has_v_mask, reps, ms);
	}
	case R_PT_I32: {
		Semiring<operators::add<int>, operators::mul<int>, identities::zero, identities::one> r;
		return mxv_ring<int>(r, descr, vxm_form, m, n, nnz, I, J, V, u, u_assigned, u_mask,
			u_mask_assigned, has_u_mask, v, v_assigned, v_mask, v_mask_assigned, has_v_mask, reps, ms);
	}
	case R_PLUS_RIGHTIF_U64: {  // interfaces/pregel.hpp:381-386
		Semiring<operators::add<size_t>, operators::right_assign_if<bool, size_t, size_t>,
			identities::zero, identities::logical_true> r;
		return mxv_ring<size_t>(r, descr, vxm_form, m, n, nnz, I, J, V, u, u_assigned, u_mask,
			u_mask_assigned, has_u_mask, v, v_assigned, v_mask, v_mask_assigned, has_v_mask, reps, ms);
	}
	case R_MAX_LEFTIF_U64: {  // pregel.hpp:714-720 under pregel_connected_components.hpp:148-151
		Semiring<operators::max<size_t>, operators::left_assign_if<size_t, bool, size_t>,
			identities::negative_infinity, identities::logical_true> r;
		return mxv_ring<size_t>(r, descr, vxm_form, m, n, nnz, I, J, V, u, u_assigned, u_mask,
			u_mask_assigned, has_u_mask, v, v_assigned, v_mask, v_mask_assigned, has_v_mask, reps, ms);
	}
	case R_TIMES_PLUS_F64: {  // tests/unit/vmxa.cpp:62-67
		Semiring<operators::mul<double>, operators::add<double>, identities::one, identities::zero> r;
		return mxv_ring<double>(r, descr, vxm_form, m, n, nnz, I, J, V, u, u_assigned, u_mask,
			u_mask_assigned, has_u_mask, v, v_assigned, v_mask, v_mask_assigned, has_v_mask, reps, ms);
	}
#endif
	}
	return int(UNSUPPORTED);
}

/* grb::algorithms::conjugate_gradient on a square FP64 matrix. */
__attribute__((visibility("default"))) int refw_cg(int64_t n, int64_t nnz, const uint32_t *I,
	const uint32_t *J, const double *V, const double *b, double *x, int64_t max_iter, double tol,
	int64_t *iterations, double *residual, double *ms) {
	ensure_init();
	const size_t N = static_cast<size_t>(n);
	Matrix<double> A(N, N, static_cast<size_t>(nnz));
	RC rc = build_matrix<double>(A, nnz, I, J, V, SEQUENTIAL);
	Vector<double> xx(N), bb(N), r(N), u(N), temp(N);
	if (rc == SUCCESS) rc = build_vector<double>(bb, n, b, nullptr);
	if (rc == SUCCESS) rc = build_vector<double>(xx, n, x, nullptr);
	if (rc != SUCCESS) return int(rc);
	size_t iters = 0;
	double res = 0;
	const double t0 = now_ms();
	rc = algorithms::conjugate_gradient(xx, A, bb, size_t(max_iter), tol, iters, res, r, u, temp);
	if (ms) *ms = now_ms() - t0;
	*iterations = int64_t(iters);
	*residual = res;
	export_vector<double>(xx, n, x, nullptr);
	return int(rc);
}

/* grb::algorithms::simple_pagerank on an FP64 link matrix. */
__attribute__((visibility("default"))) int refw_pagerank(int64_t n, int64_t nnz,
	const uint32_t *I, const uint32_t *J, const double *V, double *pr, double alpha, double conv,
	int64_t max_iter, int64_t *iterations, double *ms) {
	ensure_init();
	const size_t N = static_cast<size_t>(n);
	Matrix<double> L(N, N, static_cast<size_t>(nnz));
	RC rc = build_matrix<double>(L, nnz, I, J, V, SEQUENTIAL);
	Vector<double> p(N), pn(N), pnn(N), rs(N);
	Vector<bool> dang(N);
	if (rc != SUCCESS) return int(rc);
	size_t iters = 0;
	double quality = 0;
	const double t0 = now_ms();
	rc = algorithms::simple_pagerank<descriptors::no_operation>(p, L, pn, pnn, rs, dang, alpha,
		conv, size_t(max_iter), &iters, &quality);
	if (ms) *ms = now_ms() - t0;
	*iterations = int64_t(iters);
	export_vector<double>(p, n, pr, nullptr);
	return int(rc);
}

/* grb::algorithms::hpcg on the system build_hpcg_system makes (27-point
 * stencil on nx*ny*nz, diagonal 26, off-diagonals -1, max_levels coarser
 * levels, `colors` static colours, one pre- and one post-smoothing step),
 * one right-hand side b (NULL: b = A 1), x from zero; *ms times hpcg() alone,
 * *build_ms the system build. */
__attribute__((visibility("default"))) int refw_hpcg(int64_t nx, int64_t ny, int64_t nz,
	int64_t max_levels, int64_t colors, const double *b, double *x, int64_t max_iter, double tol,
	int64_t *iterations, double *residual, double *ms, double *build_ms) {
	ensure_init();
	using namespace grb::algorithms;
	const std::array< size_t, 3 > sizes = { size_t(nx), size_t(ny), size_t(nz) };
	hpcg_system_params< 3, double > params { sizes, 1, size_t(colors), 26.0, -1.0, 4,
		size_t(max_levels), 2 };
	std::unique_ptr< hpcg_data< double, double, double > > data;
	const double t0 = now_ms();
	RC rc = build_hpcg_system< 3, double >( data, params );
	const size_t n = size_t(nx * ny * nz);
	Semiring< operators::add< double >, operators::mul< double >, identities::zero,
		identities::one > ring;
	if (rc == SUCCESS) {
		if (b == nullptr) {
			rc = set(data->x, 1.0);
			rc = rc ? rc : set(data->b, 0.0);
			rc = rc ? rc : mxv(data->b, data->A, data->x, ring);
		} else {
			rc = build_vector<double>(data->b, int64_t(n), b, nullptr);
		}
	}
	rc = rc ? rc : set(data->x, 0.0);
	if (build_ms) *build_ms = now_ms() - t0;
	if (rc != SUCCESS) return int(rc);
	size_t iters = 0;
	double res = 0;
	const double t1 = now_ms();
	rc = hpcg(*data, true, 1, 1, size_t(max_iter), tol, iters, res);
	if (ms) *ms = now_ms() - t1;
	*iterations = int64_t(iters);
	*residual = res;
	if (x) export_vector<double>(data->x, int64_t(n), x, nullptr);
	return int(rc);
}

} // extern "C"
