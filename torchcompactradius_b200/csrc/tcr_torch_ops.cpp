// tcr_torch_ops.cpp -- the search as PyTorch operators (TORCH_LIBRARY namespace tcr_b200).
//
// A thin layer over the C ABI of libtcr_b200.so (include/tcr_b200.h): device memory comes from
// torch's caching allocator and every launch goes to torch's current CUDA stream.  Registered:
//
//   countNeighbors / buildNeighborList -- the reference's operator schemas
//     (cppSrc/neighborhood.h:102-124, registered at cppSrc/cppWrapper.cpp:38-40), so a caller that
//     binds torch.ops.torchCompactRadius_cuda.* (compactHashing/cppWrapper.py:10-65) can bind
//     torch.ops.tcr_b200.* instead.  The arguments mean what they mean there: sortedPositions /
//     sortedSupport are the reference cloud in the order of the caller's hash map, the returned
//     columns index that order.  The engine builds its own structure over sortedPositions from the
//     same positions, supports, domain, periodicity and hashMapLength (its cell size follows the
//     reference's compute_h of the largest support); hashTable, numCells, cellTable, qMin and hCell
//     are accepted for the schema and not read.  Only searchRange 1 (the 3^d stencil every
//     reference caller uses) is supported.
//   radiusSearch -- the fused search: structure, count and emit in one call, one host sync for the
//     pair count; returns (row, col, offsets) with columns in the reference cloud's input order.
//   buildStructure / radiusSearchWithStructure -- the same split in two for structure reuse
//     (many query sets against one reference cloud, the reference's CompactHashMap reuse).
//   radiusSearchBatched -- independent clouds in one set of launches (the batched engine): the
//     clouds are consecutive segments of the position tensors, given by their sizes.
#include <torch/library.h>
#include <ATen/ATen.h>
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>

#include <cstring>
#include <optional>
#include <string>
#include <tuple>
#include <vector>

#include "tcr_b200.h"

namespace {

using at::Tensor;

void check_rc(int rc, const char* what) {
    TORCH_CHECK(rc == TCR_OK, what, " failed: ", tcr_last_error());
}

int mode_of(const std::string& m) {
    if (m == "gather") return TCR_GATHER;
    if (m == "scatter") return TCR_SCATTER;
    if (m == "symmetric") return TCR_SYMMETRIC;
    if (m == "superSymmetric") return TCR_SUPERSYMMETRIC;
    TORCH_CHECK(false, "mode must be gather, scatter, symmetric or superSymmetric (got ", m, ")");
    return -1;
}

Tensor positions(const Tensor& x, const char* what) {
    TORCH_CHECK(x.is_cuda(), what, " must be a CUDA tensor");
    TORCH_CHECK(x.dim() == 2 && x.size(1) >= 1 && x.size(1) <= 3, what, " must be [n, dim] with dim 1..3");
    return x.to(at::kFloat).contiguous();
}

Tensor supports(const std::optional<Tensor>& h, int64_t n, const char* what) {
    if (!h.has_value() || !h->defined()) return Tensor();
    TORCH_CHECK(h->is_cuda(), what, " must be a CUDA tensor");
    TORCH_CHECK(h->numel() == n, what, " must hold one support per point");
    return h->to(at::kFloat).contiguous().reshape({n});
}

// The search descriptor and the tensors it points into (kept alive with it).
struct Search {
    tcr_search_desc d;
    Tensor xq, hq, xr, hr;
};

void fill_domain(tcr_search_desc& d, int dim, const Tensor& minDomain, const Tensor& maxDomain,
                 const Tensor& periodicity) {
    const Tensor lo = minDomain.detach().to(at::kCPU, at::kDouble).reshape({-1});
    const Tensor hi = maxDomain.detach().to(at::kCPU, at::kDouble).reshape({-1});
    const Tensor per = periodicity.detach().to(at::kCPU, at::kBool).reshape({-1});
    TORCH_CHECK(lo.numel() == dim && hi.numel() == dim, "the domain must have one extent per dimension");
    TORCH_CHECK(per.numel() == dim || per.numel() == 1, "periodicity must have one entry per dimension");
    d.periodic_mask = 0;
    for (int k = 0; k < 3; ++k) {
        d.domain_min[k] = k < dim ? (float)lo[k].item<double>() : 0.0f;
        d.domain_max[k] = k < dim ? (float)hi[k].item<double>() : 1.0f;
        if (k < dim && per[per.numel() == 1 ? 0 : k].item<bool>()) d.periodic_mask |= 1 << k;
    }
}

Search make_search(const Tensor& queryPositions, const std::optional<Tensor>& querySupport,
                   const Tensor& referencePositions, const std::optional<Tensor>& referenceSupport,
                   const Tensor& minDomain, const Tensor& maxDomain, const Tensor& periodicity,
                   int64_t hashMapLength, const std::string& mode, bool selfSearch) {
    Search s;
    std::memset(&s.d, 0, sizeof(s.d));
    s.xq = positions(queryPositions, "queryPositions");
    s.xr = selfSearch ? s.xq : positions(referencePositions, "referencePositions");
    TORCH_CHECK(s.xq.size(1) == s.xr.size(1), "query and reference clouds have different dimensions");
    TORCH_CHECK(s.xq.device() == s.xr.device(), "query and reference clouds are on different devices");
    const int dim = (int)s.xq.size(1);
    s.hq = supports(querySupport, s.xq.size(0), "querySupport");
    s.hr = selfSearch ? s.hq : supports(referenceSupport, s.xr.size(0), "referenceSupport");
    tcr_search_desc& d = s.d;
    d.dim = dim;
    d.mode = mode_of(mode);
    d.self_search = selfSearch ? 1 : 0;
    fill_domain(d, dim, minDomain, maxDomain, periodicity);
    d.hash_map_length = hashMapLength;
    d.n_query = s.xq.size(0);
    d.n_ref = s.xr.size(0);
    d.query_pos = d.n_query ? s.xq.data_ptr<float>() : nullptr;
    d.ref_pos = d.n_ref ? s.xr.data_ptr<float>() : nullptr;
    d.query_sup = s.hq.defined() && d.n_query ? s.hq.data_ptr<float>() : nullptr;
    d.ref_sup = s.hr.defined() && d.n_ref ? s.hr.data_ptr<float>() : nullptr;
    return s;
}

Tensor bytes_on(const Tensor& like, int64_t n) {
    return at::empty({std::max<int64_t>(n, 1)}, like.options().dtype(at::kByte));
}

// Count phase: offsets [nq+1], optional indptr/rowEntries; returns the info block (host).
std::vector<int64_t> count_phase(const Search& s, const Tensor& structure, const Tensor& scratch, const Tensor& stage,
                                 const Tensor& offsets, int32_t* indptr, int64_t* rowEntries, cudaStream_t st) {
    Tensor info = at::zeros({8}, at::TensorOptions().dtype(at::kLong).pinned_memory(true));
    check_rc(tcr_count(&s.d, structure.data_ptr(), scratch.data_ptr(), scratch.numel(),
                       stage.defined() ? stage.data_ptr<int32_t>() : nullptr, stage.defined() ? stage.numel() : 0,
                       offsets.data_ptr<int64_t>(), indptr, rowEntries, info.data_ptr<int64_t>(), st),
             "tcr_count");
    C10_CUDA_CHECK(cudaStreamSynchronize(st));
    std::vector<int64_t> out(info.data_ptr<int64_t>(), info.data_ptr<int64_t>() + 8);
    TORCH_CHECK(out[1] == 0, out[1], " cloud(s) have no valid cell grid for their domain and support (the support "
                "is not smaller than the domain extent, or a support/domain value is not finite)");
    return out;
}

// Structure, count and emit of one search; col in the reference cloud's input order.
std::tuple<Tensor, Tensor, Tensor> run_search(const Search& s, const Tensor* prebuilt) {
    const c10::cuda::CUDAGuard guard(s.xq.device());
    cudaStream_t st = at::cuda::getCurrentCUDAStream();
    int64_t s_bytes = 0, w_bytes = 0;
    check_rc(tcr_search_sizes(s.d.n_query, s.d.n_ref, s.d.dim, &s_bytes, &w_bytes), "tcr_search_sizes");
    Tensor structure;
    Tensor scratch = bytes_on(s.xq, w_bytes);
    if (prebuilt) {
        TORCH_CHECK(prebuilt->numel() >= s_bytes && prebuilt->is_cuda(),
                    "the structure was built for a different reference cloud");
        structure = *prebuilt;
    } else {
        structure = bytes_on(s.xq, s_bytes);
        check_rc(tcr_build_structure(&s.d, structure.data_ptr(), s_bytes, scratch.data_ptr(), w_bytes, st),
                 "tcr_build_structure");
    }
    const int64_t nq = s.d.n_query;
    Tensor offsets = at::empty({nq + 1}, s.xq.options().dtype(at::kLong));
    // the staging list: 96 words per query covers the records of dense 3D clouds; units that do
    // not fit are tested again by the emit (slower, never wrong)
    Tensor stage = at::empty({std::min<int64_t>(96 * nq + 65536, 0x7fffffff)}, s.xq.options().dtype(at::kInt));
    const std::vector<int64_t> info = count_phase(s, structure, scratch, stage, offsets, nullptr, nullptr, st);
    const int64_t total = info[0];
    Tensor row = at::empty({total}, s.xq.options().dtype(at::kLong));
    Tensor col = at::empty({total}, s.xq.options().dtype(at::kLong));
    if (total > 0)
        check_rc(tcr_emit(&s.d, structure.data_ptr(), scratch.data_ptr(), w_bytes, stage.data_ptr<int32_t>(),
                          offsets.data_ptr<int64_t>(), row.data_ptr<int64_t>(), col.data_ptr<int64_t>(), total, st),
                 "tcr_emit");
    return {row, col, offsets};
}

// ---- the reference's operator schemas --------------------------------------------------------

Search reference_args(const Tensor& queryPositions, const Tensor& querySupport, int64_t searchRange,
                      const Tensor& sortedPositions, const Tensor& sortedSupport, int64_t hashMapLength,
                      const Tensor& maxDomain, const Tensor& minDomain, const Tensor& periodicity,
                      const std::string& mode) {
    TORCH_CHECK(searchRange == 1, "tcr_b200 supports searchRange 1 (the 3^d stencil), got ", searchRange);
    return make_search(queryPositions, querySupport, sortedPositions, sortedSupport, minDomain, maxDomain,
                       periodicity, hashMapLength, mode, false);
}

Tensor countNeighbors(Tensor queryPositions, Tensor querySupport, int64_t searchRange, Tensor sortedPositions,
                      Tensor sortedSupport, Tensor hashTable, int64_t hashMapLength, Tensor numCells,
                      Tensor cellTable, Tensor qMin, double hCell, Tensor maxDomain, Tensor minDomain,
                      Tensor periodicity, std::string mode, bool verbose) {
    (void)hashTable, (void)numCells, (void)cellTable, (void)qMin, (void)hCell, (void)verbose;
    const Search s = reference_args(queryPositions, querySupport, searchRange, sortedPositions, sortedSupport,
                                    hashMapLength, maxDomain, minDomain, periodicity, mode);
    const c10::cuda::CUDAGuard guard(s.xq.device());
    cudaStream_t st = at::cuda::getCurrentCUDAStream();
    int64_t s_bytes = 0, w_bytes = 0;
    check_rc(tcr_search_sizes(s.d.n_query, s.d.n_ref, s.d.dim, &s_bytes, &w_bytes), "tcr_search_sizes");
    Tensor structure = bytes_on(s.xq, s_bytes), scratch = bytes_on(s.xq, w_bytes);
    check_rc(tcr_build_structure(&s.d, structure.data_ptr(), s_bytes, scratch.data_ptr(), w_bytes, st),
             "tcr_build_structure");
    Tensor offsets = at::empty({s.d.n_query + 1}, s.xq.options().dtype(at::kLong));
    Tensor entries = at::empty({s.d.n_query}, s.xq.options().dtype(at::kLong));
    count_phase(s, structure, scratch, Tensor(), offsets, nullptr, entries.data_ptr<int64_t>(), st);
    return entries.to(at::kInt);  // the reference's int32 counters
}

std::tuple<Tensor, Tensor> buildNeighborList(Tensor neighborCounter, Tensor neighborOffsets,
                                             int64_t neighborListLength, Tensor queryPositions, Tensor querySupport,
                                             int64_t searchRange, Tensor sortedPositions, Tensor sortedSupport,
                                             Tensor hashTable, int64_t hashMapLength, Tensor numCells,
                                             Tensor cellTable, Tensor qMin, double hCell, Tensor maxDomain,
                                             Tensor minDomain, Tensor periodicity, std::string mode, bool verbose) {
    (void)neighborCounter, (void)neighborOffsets, (void)hashTable, (void)numCells, (void)cellTable, (void)qMin;
    (void)hCell, (void)verbose;
    const Search s = reference_args(queryPositions, querySupport, searchRange, sortedPositions, sortedSupport,
                                    hashMapLength, maxDomain, minDomain, periodicity, mode);
    auto res = run_search(s, nullptr);
    const Tensor& row = std::get<0>(res);
    TORCH_CHECK(row.numel() == neighborListLength, "neighborListLength ", neighborListLength,
                " differs from the ", row.numel(), " pairs found (counts from another search?)");
    return {row, std::get<1>(res)};
}

// ---- the fused and split forms ----------------------------------------------------------------

std::tuple<Tensor, Tensor, Tensor> radiusSearch(Tensor queryPositions, std::optional<Tensor> querySupport,
                                                Tensor referencePositions, std::optional<Tensor> referenceSupport,
                                                Tensor minDomain, Tensor maxDomain, Tensor periodicity,
                                                int64_t hashMapLength, std::string mode, bool selfSearch) {
    const Search s = make_search(queryPositions, querySupport, referencePositions, referenceSupport, minDomain,
                                 maxDomain, periodicity, hashMapLength, mode, selfSearch);
    return run_search(s, nullptr);
}

Tensor buildStructure(Tensor queryPositions, std::optional<Tensor> querySupport, Tensor referencePositions,
                      std::optional<Tensor> referenceSupport, Tensor minDomain, Tensor maxDomain, Tensor periodicity,
                      int64_t hashMapLength, std::string mode, bool selfSearch) {
    const Search s = make_search(queryPositions, querySupport, referencePositions, referenceSupport, minDomain,
                                 maxDomain, periodicity, hashMapLength, mode, selfSearch);
    const c10::cuda::CUDAGuard guard(s.xq.device());
    cudaStream_t st = at::cuda::getCurrentCUDAStream();
    int64_t s_bytes = 0, w_bytes = 0;
    check_rc(tcr_search_sizes(s.d.n_query, s.d.n_ref, s.d.dim, &s_bytes, &w_bytes), "tcr_search_sizes");
    Tensor structure = bytes_on(s.xq, s_bytes), scratch = bytes_on(s.xq, w_bytes);
    check_rc(tcr_build_structure(&s.d, structure.data_ptr(), s_bytes, scratch.data_ptr(), w_bytes, st),
             "tcr_build_structure");
    return structure;
}

std::tuple<Tensor, Tensor, Tensor> radiusSearchWithStructure(Tensor structure, Tensor queryPositions,
                                                             std::optional<Tensor> querySupport,
                                                             Tensor referencePositions,
                                                             std::optional<Tensor> referenceSupport,
                                                             Tensor minDomain, Tensor maxDomain, Tensor periodicity,
                                                             int64_t hashMapLength, std::string mode,
                                                             bool selfSearch) {
    const Search s = make_search(queryPositions, querySupport, referencePositions, referenceSupport, minDomain,
                                 maxDomain, periodicity, hashMapLength, mode, selfSearch);
    return run_search(s, &structure);
}

std::tuple<Tensor, Tensor, Tensor> radiusSearchBatched(Tensor queryPositions, std::optional<Tensor> querySupport,
                                                       Tensor referencePositions,
                                                       std::optional<Tensor> referenceSupport,
                                                       Tensor querySizes, Tensor referenceSizes, Tensor minDomain,
                                                       Tensor maxDomain, Tensor periodicity, int64_t hashMapLength,
                                                       std::string mode, bool selfSearch, bool localIndex) {
    const Search all = make_search(queryPositions, querySupport, referencePositions, referenceSupport, minDomain,
                                   maxDomain, periodicity, hashMapLength, mode, selfSearch);
    const Tensor nq = querySizes.detach().to(at::kCPU, at::kLong).reshape({-1});
    const Tensor nr = selfSearch ? nq : referenceSizes.detach().to(at::kCPU, at::kLong).reshape({-1});
    const int64_t C = nq.numel();
    TORCH_CHECK(C >= 1 && nr.numel() == C, "one query and one reference size per cloud");
    TORCH_CHECK(nq.sum().item<int64_t>() == all.d.n_query && nr.sum().item<int64_t>() == all.d.n_ref,
                "the cloud sizes must add up to the point counts");
    const int dim = all.d.dim;
    std::vector<tcr_cloud_desc> clouds((size_t)C);
    int64_t q0 = 0, r0 = 0;
    for (int64_t k = 0; k < C; ++k) {
        tcr_cloud_desc& c = clouds[(size_t)k];
        std::memset(&c, 0, sizeof(c));
        c.dim = dim;
        c.periodic_mask = all.d.periodic_mask;
        for (int j = 0; j < 3; ++j) {
            c.domain_min[j] = all.d.domain_min[j];
            c.domain_max[j] = all.d.domain_max[j];
        }
        c.hash_map_length = hashMapLength;
        c.n_query = nq[k].item<int64_t>();
        c.n_ref = nr[k].item<int64_t>();
        c.query_pos = all.xq.data_ptr<float>() + q0 * dim;
        c.ref_pos = all.xr.data_ptr<float>() + r0 * dim;
        c.query_sup = all.hq.defined() ? all.hq.data_ptr<float>() + q0 : nullptr;
        c.ref_sup = all.hr.defined() ? all.hr.data_ptr<float>() + r0 : nullptr;
        q0 += c.n_query;
        r0 += c.n_ref;
    }
    tcr_batch_desc b;
    std::memset(&b, 0, sizeof(b));
    b.n_clouds = (int32_t)C;
    b.mode = all.d.mode;
    b.self_search = selfSearch ? 1 : 0;
    b.local_index = localIndex ? 1 : 0;
    b.clouds = clouds.data();
    const c10::cuda::CUDAGuard guard(all.xq.device());
    cudaStream_t st = at::cuda::getCurrentCUDAStream();
    int64_t s_bytes = 0, w_bytes = 0;
    check_rc(tcr_batch_sizes(&b, &s_bytes, &w_bytes), "tcr_batch_sizes");
    Tensor structure = bytes_on(all.xq, s_bytes), scratch = bytes_on(all.xq, w_bytes);
    check_rc(tcr_batch_build_structure(&b, structure.data_ptr(), s_bytes, scratch.data_ptr(), w_bytes, st),
             "tcr_batch_build_structure");
    const int64_t n = all.d.n_query;
    Tensor offsets = at::empty({n + 1}, all.xq.options().dtype(at::kLong));
    Tensor stage = at::empty({std::min<int64_t>(96 * n + 65536, 0x7fffffff)}, all.xq.options().dtype(at::kInt));
    Tensor info = at::zeros({8}, at::TensorOptions().dtype(at::kLong).pinned_memory(true));
    check_rc(tcr_batch_count(&b, structure.data_ptr(), scratch.data_ptr(), w_bytes, stage.data_ptr<int32_t>(),
                             stage.numel(), offsets.data_ptr<int64_t>(), nullptr, nullptr, info.data_ptr<int64_t>(),
                             st),
             "tcr_batch_count");
    C10_CUDA_CHECK(cudaStreamSynchronize(st));
    TORCH_CHECK(info.data_ptr<int64_t>()[1] == 0, "a cloud has no valid cell grid for its domain and support");
    const int64_t total = info.data_ptr<int64_t>()[0];
    Tensor row = at::empty({total}, all.xq.options().dtype(at::kLong));
    Tensor col = at::empty({total}, all.xq.options().dtype(at::kLong));
    if (total > 0)
        check_rc(tcr_batch_emit(&b, structure.data_ptr(), scratch.data_ptr(), w_bytes, stage.data_ptr<int32_t>(),
                                offsets.data_ptr<int64_t>(), row.data_ptr<int64_t>(), col.data_ptr<int64_t>(), total,
                                st),
                 "tcr_batch_emit");
    return {row, col, offsets};
}

}  // namespace

TORCH_LIBRARY(tcr_b200, m) {
    m.def("countNeighbors(Tensor queryPositions, Tensor querySupport, int searchRange, Tensor sortedPositions, "
          "Tensor sortedSupport, Tensor hashTable, int hashMapLength, Tensor numCells, Tensor cellTable, "
          "Tensor qMin, float hCell, Tensor maxDomain, Tensor minDomain, Tensor periodicity, str mode, "
          "bool verbose=False) -> Tensor");
    m.def("buildNeighborList(Tensor neighborCounter, Tensor neighborOffsets, int neighborListLength, "
          "Tensor queryPositions, Tensor querySupport, int searchRange, Tensor sortedPositions, "
          "Tensor sortedSupport, Tensor hashTable, int hashMapLength, Tensor numCells, Tensor cellTable, "
          "Tensor qMin, float hCell, Tensor maxDomain, Tensor minDomain, Tensor periodicity, str mode, "
          "bool verbose=False) -> (Tensor, Tensor)");
    m.def("radiusSearch(Tensor queryPositions, Tensor? querySupport, Tensor referencePositions, "
          "Tensor? referenceSupport, Tensor minDomain, Tensor maxDomain, Tensor periodicity, int hashMapLength, "
          "str mode, bool selfSearch) -> (Tensor, Tensor, Tensor)");
    m.def("buildStructure(Tensor queryPositions, Tensor? querySupport, Tensor referencePositions, "
          "Tensor? referenceSupport, Tensor minDomain, Tensor maxDomain, Tensor periodicity, int hashMapLength, "
          "str mode, bool selfSearch) -> Tensor");
    m.def("radiusSearchWithStructure(Tensor structure, Tensor queryPositions, Tensor? querySupport, "
          "Tensor referencePositions, Tensor? referenceSupport, Tensor minDomain, Tensor maxDomain, "
          "Tensor periodicity, int hashMapLength, str mode, bool selfSearch) -> (Tensor, Tensor, Tensor)");
    m.def("radiusSearchBatched(Tensor queryPositions, Tensor? querySupport, Tensor referencePositions, "
          "Tensor? referenceSupport, Tensor querySizes, Tensor referenceSizes, Tensor minDomain, "
          "Tensor maxDomain, Tensor periodicity, int hashMapLength, str mode, bool selfSearch, "
          "bool localIndex) -> (Tensor, Tensor, Tensor)");
}

TORCH_LIBRARY_IMPL(tcr_b200, CUDA, m) {
    m.impl("countNeighbors", &countNeighbors);
    m.impl("buildNeighborList", &buildNeighborList);
    m.impl("radiusSearch", &radiusSearch);
    m.impl("buildStructure", &buildStructure);
    m.impl("radiusSearchWithStructure", &radiusSearchWithStructure);
    m.impl("radiusSearchBatched", &radiusSearchBatched);
}
