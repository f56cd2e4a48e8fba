// B200Backend: IComputeBackend over libhn_sm100.so (see hn_backend.hpp).
#include "hn_backend.hpp"

#include <cstring>
#include <stdexcept>

#include "hn_sm100.h"

namespace hn::execution {
namespace {

uint64_t mix(uint64_t h, uint64_t v) {
    h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    return h;
}

// 64-bit finaliser (splitmix64's): every input bit affects every output bit.
inline uint64_t avalanche(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Hash of n 64-bit words, in chunks of 2^16 words hashed in parallel and
// combined in chunk order (the result does not depend on the thread count).
uint64_t hash_words(const void* data, std::size_t n, uint64_t seed) {
    const auto* w = static_cast<const uint64_t*>(data);
    constexpr std::size_t kChunk = std::size_t(1) << 16;
    const std::size_t chunks = (n + kChunk - 1) / kChunk;
    std::vector<uint64_t> part(chunks);
#pragma omp parallel for schedule(static) if (chunks > 4)
    for (std::size_t c = 0; c < chunks; ++c) {
        const std::size_t e = (c + 1) * kChunk < n ? (c + 1) * kChunk : n;
        uint64_t a = seed ^ (c * 0x9e3779b97f4a7c15ull), b = ~seed;
        std::size_t k = c * kChunk;
        for (; k + 1 < e; k += 2) {  // two independent lanes
            a = avalanche(a ^ w[k]) + 0x632be59bd9b4e019ull;
            b = avalanche(b ^ w[k + 1]) + 0x8cb92ba72f3d8dd7ull;
        }
        if (k < e) a = avalanche(a ^ w[k]);
        part[c] = avalanche(a ^ (b << 1) ^ (b >> 63));
    }
    uint64_t h = avalanche(seed ^ n);
    for (uint64_t v : part) h = avalanche(h ^ v);
    return h;
}

// Hash of every value, column index and row pointer: a caller that rewrites
// any entry of a matrix whose buffers it reuses gets a new device copy (the
// reference's cache checks only the pointer and the sizes,
// gpu_backend.cpp:289-306).
uint64_t fingerprint(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
                     const std::vector<std::size_t>& row_ptr) {
    static_assert(sizeof(double) == 8 && sizeof(std::size_t) == 8, "64-bit words expected");
    uint64_t h = mix(values.size(), row_ptr.size());
    h = mix(h, hash_words(values.data(), values.size(), 0x51ed270b27f1e5a1ull));
    h = mix(h, hash_words(col_indices.data(), col_indices.size(), 0x2545f4914f6cdd1dull));
    h = mix(h, hash_words(row_ptr.data(), row_ptr.size(), 0x9fb21c651e98df25ull));
    return h;
}

}  // namespace

B200Backend::~B200Backend() { release(); }

std::string B200Backend::name() const {
    return device_name_.empty() ? std::string("CUDA(B200 sm_100a)") : "CUDA(" + device_name_ + ")";
}

void B200Backend::initialize() {
    std::lock_guard<std::mutex> lk(mutex_);
    if (initialized_) return;
    initialized_ = true;
    if (hn_init(device_) != HN_OK) {
        last_error_ = hn_last_error();
        return;
    }
    hn_device_info_t info;
    if (hn_device_info(&info) == HN_OK) device_name_ = info.name;
    available_ = true;
}

void B200Backend::release() {
    for (auto& kv : cache_) hn_csr_destroy(kv.second.h);
    cache_.clear();
    if (dev_buf_) hn_free(dev_buf_);
    dev_buf_ = nullptr;
    dev_buf_len_ = 0;
}

void B200Backend::finalize() {
    std::lock_guard<std::mutex> lk(mutex_);
    release();
}

void B200Backend::require(const char* op) const {
    if (!available_) throw std::runtime_error(std::string("B200 backend not available for ") + op + ": " + last_error_);
}

B200Backend::Resident& B200Backend::resident(const std::vector<double>& values,
                                             const std::vector<std::size_t>& col_indices,
                                             const std::vector<std::size_t>& row_ptr, std::size_t ncols) {
    const std::size_t nrows = row_ptr.size() - 1;
    const uint64_t fp = fingerprint(values, col_indices, row_ptr);
    auto it = cache_.find(values.data());
    if (it != cache_.end()) {
        Resident& r = it->second;
        if (r.nnz == values.size() && r.nrows == nrows && r.ncols >= ncols && r.fingerprint == fp) return r;
        hn_csr_destroy(r.h);
        cache_.erase(it);
    }
    std::size_t n = ncols;
    for (std::size_t c : col_indices) n = c + 1 > n ? c + 1 : n;
    Resident r;
    static_assert(sizeof(std::size_t) == sizeof(uint64_t), "size_t must be 64-bit");
    if (hn_csr_create((int64_t)nrows, (int64_t)n, reinterpret_cast<const uint64_t*>(row_ptr.data()),
                      reinterpret_cast<const uint64_t*>(col_indices.data()), values.data(), 0, &r.h) != HN_OK)
        throw std::runtime_error(std::string("B200 matrix upload failed: ") + hn_last_error());
    r.nnz = values.size();
    r.nrows = nrows;
    r.ncols = n;
    r.fingerprint = fp;
    return cache_.emplace(values.data(), r).first->second;
}

double* B200Backend::staging(std::size_t doubles) {
    if (dev_buf_len_ < doubles) {
        if (dev_buf_) hn_free(dev_buf_);
        dev_buf_ = nullptr;
        void* p = nullptr;
        if (hn_malloc(&p, doubles * 8) != HN_OK) throw std::runtime_error(hn_last_error());
        dev_buf_ = static_cast<double*>(p);
        dev_buf_len_ = doubles;
    }
    return dev_buf_;
}

void B200Backend::spmv(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
                       const std::vector<std::size_t>& row_ptr, const std::vector<double>& x, std::vector<double>& y) {
    std::lock_guard<std::mutex> lk(mutex_);
    require("spmv");
    const std::size_t nrows = row_ptr.size() >= 1 ? row_ptr.size() - 1 : 0;
    if (values.empty() || row_ptr.size() < 2) {  // gpu_backend.cpp:206-209
        y.assign(nrows, 0.0);
        return;
    }
    Resident& r = resident(values, col_indices, row_ptr, x.size());
    if (x.size() < r.ncols) throw std::runtime_error("B200 spmv: x shorter than the matrix's column count");
    y.resize(nrows);
    if (hn_spmv_host(r.h, 0, x.data(), y.data()) != HN_OK)
        throw std::runtime_error(std::string("B200 spmv failed: ") + hn_last_error());
}

void B200Backend::spmv_t(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
                         const std::vector<std::size_t>& row_ptr, std::size_t ncols, const std::vector<double>& x,
                         std::vector<double>& y) {
    std::lock_guard<std::mutex> lk(mutex_);
    require("spmv_t");
    const std::size_t nrows = row_ptr.size() >= 1 ? row_ptr.size() - 1 : 0;
    if (values.empty() || row_ptr.size() < 2) {
        y.assign(ncols, 0.0);
        return;
    }
    Resident& r = resident(values, col_indices, row_ptr, ncols);
    if (x.size() < nrows) throw std::runtime_error("B200 spmv_t: x shorter than the row count");
    std::vector<double> out(r.ncols);
    if (hn_spmv_host(r.h, 1, x.data(), out.data()) != HN_OK)
        throw std::runtime_error(std::string("B200 spmv_t failed: ") + hn_last_error());
    out.resize(ncols);
    y.swap(out);
}

void B200Backend::spmm(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
                       const std::vector<std::size_t>& row_ptr, const std::vector<double>& B, std::vector<double>& C,
                       std::size_t ncols_B) {
    std::lock_guard<std::mutex> lk(mutex_);
    require("spmm");
    const std::size_t nrows = row_ptr.size() >= 1 ? row_ptr.size() - 1 : 0;
    if (values.empty() || row_ptr.size() < 2 || ncols_B == 0) {  // gpu_backend.cpp:224-227
        C.assign(nrows * ncols_B, 0.0);
        return;
    }
    Resident& r = resident(values, col_indices, row_ptr, B.size() / ncols_B);
    if (B.size() < r.ncols * ncols_B) throw std::runtime_error("B200 spmm: B smaller than ncols x k");
    C.resize(nrows * ncols_B);
    if (hn_spmm_host(r.h, 0, B.data(), (int64_t)ncols_B, C.data()) != HN_OK)
        throw std::runtime_error(std::string("B200 spmm failed: ") + hn_last_error());
}

double B200Backend::dot(const std::vector<double>& a, const std::vector<double>& b) {
    std::lock_guard<std::mutex> lk(mutex_);
    require("dot");
    const std::size_t n = a.size() < b.size() ? a.size() : b.size();  // gpu_backend.cpp:123-126
    double* d = staging(2 * n + 1);
    double out = 0.0;
    if (hn_memcpy_h2d(d, a.data(), 8 * n, nullptr) != HN_OK || hn_memcpy_h2d(d + n, b.data(), 8 * n, nullptr) != HN_OK ||
        hn_dot((int64_t)n, d, d + n, d + 2 * n, nullptr) != HN_OK || hn_memcpy_d2h(&out, d + 2 * n, 8, nullptr) != HN_OK)
        throw std::runtime_error(std::string("B200 dot failed: ") + hn_last_error());
    return out;
}

void B200Backend::axpy(double alpha, const std::vector<double>& x, std::vector<double>& y) {
    std::lock_guard<std::mutex> lk(mutex_);
    require("axpy");
    const std::size_t n = x.size() < y.size() ? x.size() : y.size();  // gpu_backend.cpp:127-129
    double* d = staging(2 * n + 1);
    if (hn_memcpy_h2d(d, x.data(), 8 * n, nullptr) != HN_OK || hn_memcpy_h2d(d + n, y.data(), 8 * n, nullptr) != HN_OK ||
        hn_axpy((int64_t)n, alpha, d, d + n, nullptr) != HN_OK ||
        hn_memcpy_d2h(y.data(), d + n, 8 * n, nullptr) != HN_OK)
        throw std::runtime_error(std::string("B200 axpy failed: ") + hn_last_error());
}

double B200Backend::norm_inf(const std::vector<double>& v) {
    std::lock_guard<std::mutex> lk(mutex_);
    require("norm_inf");
    const std::size_t n = v.size();
    double* d = staging(n + 1);
    double out = 0.0;
    if (hn_memcpy_h2d(d, v.data(), 8 * n, nullptr) != HN_OK || hn_nrm_inf((int64_t)n, d, d + n, nullptr) != HN_OK ||
        hn_memcpy_d2h(&out, d + n, 8, nullptr) != HN_OK)
        throw std::runtime_error(std::string("B200 norm_inf failed: ") + hn_last_error());
    return out;
}

std::size_t B200Backend::device_memory() const {
    hn_device_info_t info;
    return hn_device_info(&info) == HN_OK ? info.total_mem : 0;
}

std::size_t B200Backend::free_memory() const {
    hn_device_info_t info;
    return hn_device_info(&info) == HN_OK ? info.free_mem : 0;
}

bool B200Backend::was_gpu_kernel_executed() const { return gpu_kernel_executions() > 0; }

std::size_t B200Backend::gpu_kernel_executions() const {
    uint64_t l = 0;
    hn_stats(&l, nullptr);
    return static_cast<std::size_t>(l - launches_at_reset_);
}

void B200Backend::reset_execution_stats() {
    uint64_t l = 0;
    hn_stats(&l, nullptr);
    launches_at_reset_ = l;
}

std::unique_ptr<IComputeBackend> ComputeBackendFactory::create_backend(ComputeBackendType type) {
    if (type != ComputeBackendType::CUDA && type != ComputeBackendType::AUTO)
        throw std::invalid_argument("this library provides the CUDA (B200) backend only");
    auto b = std::make_unique<B200Backend>();
    b->initialize();
    return b;
}

}  // namespace hn::execution
