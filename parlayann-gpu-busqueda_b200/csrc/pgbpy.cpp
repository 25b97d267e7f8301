// pgbpy.cpp -- _pgbpy, a pybind11 module over the C ABI for big-ann-benchmarks-style
// harnesses: the role of ParlayANN's compiled module `_ParlayANNpy` (built by the
// reference at cpu_baseline/setup.sh:81-88), whose harness loads an index from files
// and calls a batch search with numpy arrays. Everything here goes through include/pgb.h;
// no search logic lives in this file.
//
//   import _pgbpy
//   idx = _pgbpy.FlatIndex("base.i8bin", "vamana.graph", "int8", device=0)
//   ids, dists = idx.batch_search(queries, knn=10, beam_size=40, cut=1.35, limit=-1)
//   hidx = _pgbpy.HNSWIndex("base.i8bin", "model.hnsw", "int8")
//   deg, edges = _pgbpy.build_vamana(x, R=64, L=128, alpha=1.2)   # GPU construction
//   deg, edges = _pgbpy.build_hcnng(x, trees=30, leaf=1000, mst_deg=3)
//   _pgbpy.build_hnsw(x, "model.hnsw", M=32, ef_construction=128)
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <tuple>

#include "../../include/pgb.h"

namespace py = pybind11;

namespace {

void check(pgb_status s) {
    if (s != PGB_OK) throw std::runtime_error(std::string(pgb_status_string(s)) + ": " + pgb_last_error());
}

pgb_elem elem_of(const std::string& dtype) {
    if (dtype == "int8") return PGB_INT8;
    if (dtype == "uint8") return PGB_UINT8;
    throw std::invalid_argument("dtype must be 'int8' or 'uint8'");
}

class Index {
  public:
    Index(pgb_index* h, pgb_elem e) : h_(h), elem_(e) { check(pgb_index_get_info(h_, &info_)); }
    ~Index() { pgb_index_destroy(h_); }
    Index(const Index&) = delete;
    Index& operator=(const Index&) = delete;

    // (ids uint32 [nq, knn], dists int32 [nq, knn]); the searcher is prepared for this
    // batch and released after it (the reference's preparar / lanzar / liberar)
    py::tuple batch_search(py::array queries, uint32_t knn, uint32_t beam_size, double cut,
                           int64_t limit, uint32_t degree_limit, bool stats) {
        auto q = py::array::ensure(queries, py::array::c_style);
        if (!q || q.ndim() != 2) throw std::invalid_argument("queries: a 2-d array");
        if ((uint32_t)q.shape(1) != info_.dim) throw std::invalid_argument("queries: wrong dimension");
        if (q.itemsize() != 1) throw std::invalid_argument("queries: 8-bit elements");
        const uint32_t nq = (uint32_t)q.shape(0);
        py::array_t<uint32_t> ids({(py::ssize_t)nq, (py::ssize_t)knn});
        py::array_t<int32_t> dists({(py::ssize_t)nq, (py::ssize_t)knn});
        py::array_t<int32_t> st({(py::ssize_t)nq, (py::ssize_t)4});
        auto result = [&]() -> py::tuple {
            if (stats) return py::make_tuple(ids, dists, st);
            return py::make_tuple(ids, dists);
        };
        if (nq == 0) return result();
        pgb_query_params p{};
        p.k = knn;
        p.beam_size = beam_size;
        p.cut = cut;
        p.limit = limit;
        p.degree_limit = degree_limit;
        p.exclude_query_id = 0;  // harness queries are not base points
        pgb_searcher* s = nullptr;
        pgb_status rc;
        {
            py::gil_scoped_release nogil;
            rc = pgb_searcher_create(h_, nq, &p, &s);
            if (rc == PGB_OK)
                rc = pgb_searcher_search_host(s, q.data(), nq, info_.dim, ids.mutable_data(),
                                              dists.mutable_data(),
                                              reinterpret_cast<pgb_query_stats*>(st.mutable_data()));
            pgb_searcher_destroy(s);
        }
        check(rc);
        return result();
    }

    uint32_t n() const { return info_.n_points; }
    uint32_t dim() const { return info_.dim; }
    uint64_t device_bytes() const { return info_.device_bytes; }

  private:
    pgb_index* h_;
    pgb_elem elem_;
    pgb_index_info info_{};
};

Index* load_flat(const std::string& vectors, const std::string& graph, const std::string& dtype, int device) {
    pgb_index* h = nullptr;
    const pgb_elem e = elem_of(dtype);
    check(pgb_index_load_flat(device, vectors.c_str(), e, graph.c_str(), &h));
    return new Index(h, e);
}

Index* load_hnsw(const std::string& vectors, const std::string& model, const std::string& dtype, int device) {
    pgb_index* h = nullptr;
    const pgb_elem e = elem_of(dtype);
    check(pgb_index_load_hnsw(device, vectors.c_str(), e, model.c_str(), &h));
    return new Index(h, e);
}

py::tuple build_vamana(py::array x, uint32_t R, uint32_t L, float alpha, int passes, uint64_t seed,
                       int device) {
    auto a = py::array::ensure(x, py::array::c_style);
    if (!a || a.ndim() != 2 || a.itemsize() != 1) throw std::invalid_argument("x: a 2-d 8-bit array");
    const pgb_elem e = a.dtype().kind() == 'i' ? PGB_INT8 : PGB_UINT8;
    const uint32_t n = (uint32_t)a.shape(0), d = (uint32_t)a.shape(1);
    py::array_t<uint32_t> deg(n);
    py::array_t<uint32_t> adj({(py::ssize_t)n, (py::ssize_t)R});
    pgb_status rc;
    {
        py::gil_scoped_release nogil;
        rc = pgb_build_vamana_gpu(device, a.data(), n, d, e, R, L, alpha, passes, seed,
                                  deg.mutable_data(), adj.mutable_data());
    }
    check(rc);
    return py::make_tuple(deg, adj);
}

py::tuple build_hcnng(py::array x, uint32_t trees, uint32_t leaf, uint32_t mst_deg, uint64_t seed,
                      int device) {
    auto a = py::array::ensure(x, py::array::c_style);
    if (!a || a.ndim() != 2 || a.itemsize() != 1) throw std::invalid_argument("x: a 2-d 8-bit array");
    const pgb_elem e = a.dtype().kind() == 'i' ? PGB_INT8 : PGB_UINT8;
    const uint32_t n = (uint32_t)a.shape(0), d = (uint32_t)a.shape(1);
    py::array_t<uint32_t> deg(n);
    py::array_t<uint32_t> adj({(py::ssize_t)n, (py::ssize_t)trees * mst_deg});
    pgb_status rc;
    {
        py::gil_scoped_release nogil;
        rc = pgb_build_hcnng_gpu(device, a.data(), n, d, e, trees, leaf, mst_deg, seed,
                                 deg.mutable_data(), adj.mutable_data());
    }
    check(rc);
    return py::make_tuple(deg, adj);
}

void build_hnsw(py::array x, const std::string& path, uint32_t M, uint32_t ef_construction, float ml,
                float alpha, uint64_t seed, int device) {
    auto a = py::array::ensure(x, py::array::c_style);
    if (!a || a.ndim() != 2 || a.itemsize() != 1) throw std::invalid_argument("x: a 2-d 8-bit array");
    const pgb_elem e = a.dtype().kind() == 'i' ? PGB_INT8 : PGB_UINT8;
    pgb_status rc;
    {
        py::gil_scoped_release nogil;
        rc = pgb_build_hnsw_gpu(device, a.data(), (uint32_t)a.shape(0), (uint32_t)a.shape(1), e, M,
                                ef_construction, ml, alpha, seed, path.c_str());
    }
    check(rc);
}

double compute_recall(py::array_t<uint32_t, py::array::c_style> gt_ids,
                      py::array_t<float, py::array::c_style> gt_dists,
                      py::array_t<uint32_t, py::array::c_style> ids, uint32_t k) {
    if (gt_ids.ndim() != 2 || gt_dists.ndim() != 2 || ids.ndim() != 2 || gt_ids.shape(0) != ids.shape(0) ||
        gt_dists.shape(0) != gt_ids.shape(0) || gt_dists.shape(1) != gt_ids.shape(1))
        throw std::invalid_argument("recall: shapes");
    return pgb_recall(gt_ids.data(), gt_dists.data(), (uint32_t)gt_ids.shape(0), (uint32_t)gt_ids.shape(1),
                      ids.data(), (uint32_t)ids.shape(1)) ;
}

}  // namespace

PYBIND11_MODULE(_pgbpy, m) {
    m.doc() = "B200 graph beam search (ParlayANN search API) for big-ann-benchmarks-style harnesses";
    py::class_<Index>(m, "Index")
        .def("batch_search", &Index::batch_search, py::arg("queries"), py::arg("knn"),
             py::arg("beam_size"), py::arg("cut") = 1.35, py::arg("limit") = -1,
             py::arg("degree_limit") = 0, py::arg("stats") = false,
             "(ids, dists[, stats]) of the k nearest found for each query row")
        .def_property_readonly("n", &Index::n)
        .def_property_readonly("dim", &Index::dim)
        .def_property_readonly("device_bytes", &Index::device_bytes);
    m.def("FlatIndex", &load_flat, py::arg("vectors_path"), py::arg("graph_path"),
          py::arg("dtype") = "int8", py::arg("device") = 0, py::return_value_policy::take_ownership,
          "flat graph (Vamana / HCNNG / PyNNDescent file) over .i8bin / .u8bin vectors");
    m.def("HNSWIndex", &load_hnsw, py::arg("vectors_path"), py::arg("model_path"),
          py::arg("dtype") = "int8", py::arg("device") = 0, py::return_value_policy::take_ownership,
          "HNSW v3 model over .i8bin / .u8bin vectors");
    m.def("build_vamana", &build_vamana, py::arg("x"), py::arg("R") = 64, py::arg("L") = 128,
          py::arg("alpha") = 1.2f, py::arg("passes") = 1, py::arg("seed") = 0, py::arg("device") = 0,
          "GPU Vamana construction: (degrees [n], adjacency [n, R] padded with 0xFFFFFFFF)");
    m.def("build_hcnng", &build_hcnng, py::arg("x"), py::arg("trees") = 30, py::arg("leaf") = 1000,
          py::arg("mst_deg") = 3, py::arg("seed") = 0, py::arg("device") = 0,
          "GPU HCNNG construction: (degrees [n], adjacency [n, trees * mst_deg])");
    m.def("build_hnsw", &build_hnsw, py::arg("x"), py::arg("path"), py::arg("M") = 32,
          py::arg("ef_construction") = 128, py::arg("ml") = 0.36f, py::arg("alpha") = 0.83f,
          py::arg("seed") = 0, py::arg("device") = 0,
          "GPU HNSW construction, written to an HNSW v3 model file at path");
    m.def("compute_recall", &compute_recall, py::arg("gt_ids"), py::arg("gt_dists"), py::arg("ids"),
          py::arg("k"), "recall@k with distance ties (the reference's calcularRecall)");
}
