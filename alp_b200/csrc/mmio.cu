// MatrixMarket ingest straight to the device.
//
// ALP reads a MatrixMarket file through grb::utils::MatrixFileReader
// (include/graphblas/utils/parser/matrixFileReader.hpp, matrixFileIterator.hpp;
// src/graphblas/utils/hpparser.c) and hands its nonzero iterator to
// buildMatrixUnique, which builds both orientations on one core.  Here the
// file is parsed on the host by all cores at once (the text split into
// line-aligned chunks, one thread per chunk, chunks concatenated in file
// order), the triples go to the device in one copy each, and the device
// builds the storage (alpb_coo_to_crs, alpb_crs_transpose).
//
// The triples come out in the order ALP's iterator yields them: file order,
// 1-based indices made 0-based, and for a symmetric file every off-diagonal
// entry followed at once by its mirror (matrixFileIterator.hpp:411-434); a
// pattern file's entries take the value 1.
#include "common.cuh"

#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

namespace alpb {

struct MmHeader {
	bool pattern = false, integer = false, symmetric = false;
	int64_t m = 0, n = 0, entries = 0;
	size_t data_begin = 0;   // offset of the first entry line
};

// Banner, comments and size line.
static int mm_header(const std::vector<char> &buf, MmHeader &h) {
	const char *p = buf.data(), *end = p + buf.size();
	const char *eol = static_cast<const char *>(memchr(p, '\n', size_t(end - p)));
	if (!eol) eol = end;
	const std::string banner(p, size_t(eol - p));
	std::vector<std::string> w;
	for (size_t i = 0; i < banner.size();) {
		while (i < banner.size() && isspace(static_cast<unsigned char>(banner[i]))) ++i;
		size_t j = i;
		while (j < banner.size() && !isspace(static_cast<unsigned char>(banner[j]))) ++j;
		if (j > i) w.push_back(banner.substr(i, j - i));
		i = j;
	}
	for (auto &t : w)
		for (auto &c : t) c = char(std::tolower(static_cast<unsigned char>(c)));
	ALPB_CHECK(w.size() >= 5 && w[0] == "%%matrixmarket" && w[1] == "matrix" &&
		w[2] == "coordinate", ALPB_ILLEGAL,
		"alpb_mm_read: not a MatrixMarket coordinate file");
	ALPB_CHECK(w[3] == "real" || w[3] == "integer" || w[3] == "pattern", ALPB_UNSUPPORTED,
		"alpb_mm_read: field '%s' (real, integer and pattern are read)", w[3].c_str());
	ALPB_CHECK(w[4] == "general" || w[4] == "symmetric", ALPB_UNSUPPORTED,
		"alpb_mm_read: symmetry '%s' (general and symmetric are read)", w[4].c_str());
	h.pattern = w[3] == "pattern";
	h.integer = w[3] == "integer";
	h.symmetric = w[4] == "symmetric";
	p = eol < end ? eol + 1 : end;
	while (p < end && *p == '%') {                    // comments
		const char *e = static_cast<const char *>(memchr(p, '\n', size_t(end - p)));
		p = e ? e + 1 : end;
	}
	char *q = nullptr;
	h.m = strtoll(p, &q, 10);
	h.n = strtoll(q, &q, 10);
	h.entries = strtoll(q, &q, 10);
	ALPB_CHECK(q != p && h.m > 0 && h.n > 0 && h.entries >= 0 && h.m <= 0xFFFFFFFFll &&
		h.n <= 0xFFFFFFFFll, ALPB_ILLEGAL, "alpb_mm_read: bad size line");
	const char *e = static_cast<const char *>(memchr(q, '\n', size_t(end - q)));
	h.data_begin = size_t((e ? e + 1 : end) - buf.data());
	return ALPB_SUCCESS;
}

struct MmChunk {
	std::vector<uint32_t> I, J;
	std::vector<double> V;
	int64_t bad_line = 0;    // 1-based index within the chunk of a malformed line; 0: none
};

// Entry lines of [p, end): "i j [v]".
static void mm_parse_chunk(const char *p, const char *end, const MmHeader &h, MmChunk &out) {
	int64_t line = 0;
	while (p < end) {
		const char *eol = static_cast<const char *>(memchr(p, '\n', size_t(end - p)));
		if (!eol) eol = end;
		++line;
		const char *s = p;
		while (s < eol && isspace(static_cast<unsigned char>(*s))) ++s;
		if (s < eol && *s != '%') {
			char *q = nullptr;
			const unsigned long long i = strtoull(s, &q, 10);
			char *q2 = nullptr;
			const unsigned long long j = strtoull(q, &q2, 10);
			double v = 1.0;
			bool ok = q != s && q2 != q && i >= 1 && j >= 1 && i <= uint64_t(h.m) &&
				j <= uint64_t(h.n);
			if (ok && !h.pattern) {
				char *q3 = nullptr;
				v = strtod(q2, &q3);
				ok = q3 != q2;
			}
			if (!ok) {
				if (!out.bad_line) out.bad_line = line;
			} else {
				out.I.push_back(uint32_t(i - 1));
				out.J.push_back(uint32_t(j - 1));
				out.V.push_back(v);
				if (h.symmetric && i != j) {              // the mirror, right after
					out.I.push_back(uint32_t(j - 1));
					out.J.push_back(uint32_t(i - 1));
					out.V.push_back(v);
				}
			}
		}
		p = eol < end ? eol + 1 : end;
	}
}

template <class T>
__global__ void k_mm_values(const double *in, T *out, int64_t n) {
	for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
		 k += int64_t(gridDim.x) * blockDim.x)
		out[k] = std::is_same<T, uint8_t>::value ? T(in[k] != 0.0 ? 1 : 0) : T(in[k]);
}

} // namespace alpb

using namespace alpb;

extern "C" int alpb_mm_read(const char *path, int value_type, int64_t *m, int64_t *n,
	int64_t *nnz, uint32_t **rows, uint32_t **cols, void **values, void *stream) {
	ALPB_CHECK(path && m && n && nnz && rows && cols && values, ALPB_ILLEGAL,
		"alpb_mm_read: null argument");
	ALPB_CHECK(value_type == ALPB_FP64 || value_type == ALPB_INT32 || value_type == ALPB_BOOL ||
		value_type == ALPB_VOID, ALPB_UNSUPPORTED, "alpb_mm_read: value type %d", value_type);
	*rows = *cols = nullptr;
	*values = nullptr;
	*m = *n = *nnz = 0;
	FILE *f = fopen(path, "rb");
	ALPB_CHECK(f != nullptr, ALPB_ILLEGAL, "alpb_mm_read: cannot open %s: %s", path,
		strerror(errno));
	std::vector<char> buf;
	fseek(f, 0, SEEK_END);
	const long size = ftell(f);
	fseek(f, 0, SEEK_SET);
	if (size > 0) {
		buf.resize(size_t(size));
		const size_t got = fread(buf.data(), 1, size_t(size), f);
		buf.resize(got);
	}
	fclose(f);
	MmHeader h;
	int rc = mm_header(buf, h);
	if (rc != ALPB_SUCCESS) return rc;
	// line-aligned chunks, one thread each
	const size_t begin = h.data_begin, total = buf.size() - begin;
	unsigned nt = std::thread::hardware_concurrency();
	if (nt < 1) nt = 1;
	if (nt > 64) nt = 64;
	if (total < (size_t(1) << 20)) nt = 1;
	std::vector<size_t> cut(nt + 1, buf.size());
	cut[0] = begin;
	for (unsigned t = 1; t < nt; ++t) {
		size_t c = begin + total * t / nt;
		if (c < cut[t - 1]) c = cut[t - 1];
		while (c < buf.size() && buf[c - 1] != '\n') ++c;
		cut[t] = c;
	}
	std::vector<MmChunk> chunks(nt);
	std::vector<std::thread> pool;
	for (unsigned t = 0; t < nt; ++t)
		pool.emplace_back([&, t] {
			mm_parse_chunk(buf.data() + cut[t], buf.data() + cut[t + 1], h, chunks[t]);
		});
	for (auto &th : pool) th.join();
	int64_t count = 0;
	for (unsigned t = 0; t < nt; ++t) {
		ALPB_CHECK(chunks[t].bad_line == 0, ALPB_ILLEGAL,
			"alpb_mm_read: malformed entry line in %s (chunk %u, line %lld of it)", path, t,
			(long long) chunks[t].bad_line);
		count += int64_t(chunks[t].I.size());
	}
	const int64_t stored = h.symmetric ? -1 : h.entries;
	ALPB_CHECK(stored < 0 || count == stored, ALPB_ILLEGAL,
		"alpb_mm_read: %lld entries read, the size line announces %lld", (long long) count,
		(long long) stored);
	cudaStream_t s = as_stream(stream);
	uint32_t *dI = nullptr, *dJ = nullptr;
	double *dV = nullptr;
	void *out_v = nullptr;
	const size_t bytes4 = size_t(count > 0 ? count : 1) * 4;
	bool ok = cudaMalloc(&dI, bytes4) == cudaSuccess && cudaMalloc(&dJ, bytes4) == cudaSuccess;
	if (ok && value_type != ALPB_VOID) {
		ok = cudaMalloc(&dV, size_t(count > 0 ? count : 1) * 8) == cudaSuccess &&
			cudaMalloc(&out_v, size_t(count > 0 ? count : 1) * type_size(value_type)) ==
				cudaSuccess;
	}
	if (!ok) {
		cudaGetLastError();
		cudaFree(dI);
		cudaFree(dJ);
		cudaFree(dV);
		cudaFree(out_v);
		set_error("alpb_mm_read: out of device memory for %lld entries", (long long) count);
		return ALPB_OUTOFMEM;
	}
	int64_t at = 0;
	for (unsigned t = 0; t < nt; ++t) {
		const size_t k = chunks[t].I.size();
		if (k == 0) continue;
		ALPB_CUDA(cudaMemcpyAsync(dI + at, chunks[t].I.data(), k * 4, cudaMemcpyHostToDevice, s));
		ALPB_CUDA(cudaMemcpyAsync(dJ + at, chunks[t].J.data(), k * 4, cudaMemcpyHostToDevice, s));
		if (dV)
			ALPB_CUDA(cudaMemcpyAsync(dV + at, chunks[t].V.data(), k * 8, cudaMemcpyHostToDevice, s));
		at += int64_t(k);
	}
	if (dV && count > 0) {
		switch (value_type) {
		case ALPB_FP64: k_mm_values<double><<<grid_for(count, 256), 256, 0, s>>>(dV,
			static_cast<double *>(out_v), count); break;
		case ALPB_INT32: k_mm_values<int32_t><<<grid_for(count, 256), 256, 0, s>>>(dV,
			static_cast<int32_t *>(out_v), count); break;
		default: k_mm_values<uint8_t><<<grid_for(count, 256), 256, 0, s>>>(dV,
			static_cast<uint8_t *>(out_v), count); break;
		}
		ALPB_LAUNCHED();
	}
	ALPB_CUDA(cudaStreamSynchronize(s));   // the host chunks go out of scope below
	cudaFree(dV);
	*m = h.m;
	*n = h.n;
	*nnz = count;
	*rows = dI;
	*cols = dJ;
	*values = out_v;
	return ALPB_SUCCESS;
}
