// pymodule.cpp -- the drop-in `wtivo_gpupr` Python module.
//
// Same exports, argument names, defaults, validation order, error text and
// return tuples as the reference module built from
// native/gpupr/wtivo_gpupr_bindings.cpp:579-600:
//   graph_cut_fast(vertices, tets_cuda, neighbors_cuda, labels, fill_T,
//                  threads=16, global_relabel_period=1024,
//                  max_rounds=2000000, local_steps=8)        -> 18-tuple
//   graph_cut_gpupr_fast_v630(...)  (alias)
//   surface_extraction_topology_cuda(labels, vertices, tets_cuda,
//                                    neighbors_cuda, threads=16) -> (V, F)
// PyTorch tensors appear only here: they are inspected through their Python
// attributes (is_cuda, dtype, shape, data_ptr), so this module links only
// libwtivo_gpupr.so and never libtorch.  All work goes through the C ABI of
// include/wtivo_gpupr.h.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>

#include <sys/mman.h>

#include "wtivo_gpupr.h"

namespace py = pybind11;

namespace {

thread_local gpupr_cut_stats t_last{};

[[noreturn]] void raise_status(gpupr_status st)
{
    std::string msg = gpupr_last_error();
    if (msg.empty()) msg = gpupr_status_string(st);
    throw std::runtime_error(msg);
}

bool verbose()
{
    const char* v = std::getenv("WTIVO_GPUPR_VERBOSE");
    return v && v[0] && v[0] != '0';
}

struct Topo {
    uintptr_t tets = 0, nbrs = 0;
    int64_t n = 0;
    int device = 0;
};

// bindings.cpp:116-125 (graph cut) / :412-418 (surface, one message)
Topo check_topology(const py::object& tets, const py::object& nbr, bool surface)
{
    py::module_ torch = py::module_::import("torch");
    py::object Tensor = torch.attr("Tensor");
    if (!py::isinstance(tets, Tensor) || !py::isinstance(nbr, Tensor))
        throw py::type_error("tets_cuda and neighbors_cuda must be torch.Tensor objects");
    const char* smsg = "tets/neighbors must be contiguous CUDA int32 Nx4 with same N";
    if (!tets.attr("is_cuda").cast<bool>() || !nbr.attr("is_cuda").cast<bool>())
        throw std::runtime_error(surface ? smsg : "tets/neighbors must be CUDA tensors");
    py::object i32 = torch.attr("int32");
    if (!py::object(tets.attr("dtype")).equal(i32) || !py::object(nbr.attr("dtype")).equal(i32))
        throw std::runtime_error(surface ? smsg : "tets/neighbors must be int32");
    if (!tets.attr("is_contiguous")().cast<bool>() || !nbr.attr("is_contiguous")().cast<bool>())
        throw std::runtime_error(surface ? smsg : "tets/neighbors must be contiguous");
    if (tets.attr("dim")().cast<int64_t>() != 2 || nbr.attr("dim")().cast<int64_t>() != 2 ||
        tets.attr("size")(1).cast<int64_t>() != 4 || nbr.attr("size")(1).cast<int64_t>() != 4 ||
        tets.attr("size")(0).cast<int64_t>() != nbr.attr("size")(0).cast<int64_t>())
        throw std::runtime_error(surface ? smsg : "tets/neighbors must be Nx4 and same N");
    Topo t;
    t.n = tets.attr("size")(0).cast<int64_t>();
    t.tets = tets.attr("data_ptr")().cast<uintptr_t>();
    t.nbrs = nbr.attr("data_ptr")().cast<uintptr_t>();
    t.device = tets.attr("device").attr("index").cast<int>();
    return t;
}

void* current_stream(int device)
{
    py::module_ torch = py::module_::import("torch");
    py::object s = torch.attr("cuda").attr("current_stream")(device);
    return reinterpret_cast<void*>(s.attr("cuda_stream").cast<uintptr_t>());
}

using F64 = py::array_t<double, py::array::c_style | py::array::forcecast>;

// The returned labels (one byte per tet, 80 MB at benchmark size).  Large
// outputs live in page-locked memory from PyTorch's caching host allocator
// (the numpy array holds the tensor as its base), so the device writes them
// with one DMA copy instead of through pinned staging chunks and a host
// memcpy, and the block is reused by the next call once the caller drops the
// array.  Where pinned memory cannot be had, memory aligned to 2 MiB and
// advised for huge pages: the staged copy then touches a few dozen pages
// instead of ~20,000 fresh 4 KiB ones.
py::array_t<std::uint8_t> label_array(std::uint64_t n)
{
    const std::size_t huge = 2u << 20;
    if (n < 2 * huge) return py::array_t<std::uint8_t>(static_cast<py::ssize_t>(n));
    try {
        py::module_ torch = py::module_::import("torch");
        py::object t = torch.attr("empty")(py::int_(n), py::arg("dtype") = torch.attr("uint8"),
                                           py::arg("pin_memory") = true);
        py::array_t<std::uint8_t> a = py::array_t<std::uint8_t>::ensure(t.attr("numpy")());
        if (a && a.ndim() == 1 && static_cast<std::uint64_t>(a.shape(0)) == n && a.writeable()) return a;
    } catch (const py::error_already_set&) {
        // no pinned memory here (no device, or it ran out): fall back below
    }
    const std::size_t bytes = (static_cast<std::size_t>(n) + huge - 1) / huge * huge;
    void* p = nullptr;
    if (posix_memalign(&p, huge, bytes) != 0 || !p) throw std::bad_alloc();
    madvise(p, bytes, MADV_HUGEPAGE);   // advice only: ignored where unsupported
    py::capsule owner(p, [](void* q) { std::free(q); });
    return py::array_t<std::uint8_t>({static_cast<py::ssize_t>(n)}, {static_cast<py::ssize_t>(1)},
                                     static_cast<std::uint8_t*>(p), owner);
}
using U8 = py::array_t<std::uint8_t, py::array::c_style | py::array::forcecast>;

py::tuple graph_cut_fast(F64 vertices, py::object tets_cuda, py::object nbr_cuda, U8 labels,
                         double fill_T, int threads, int global_relabel_period,
                         std::uint64_t max_rounds, int local_steps)
{
    // bindings.cpp:114-132, in the same order
    if (vertices.ndim() != 2 || vertices.shape(1) != 3)
        throw std::runtime_error("vertices must be float64 Nx3");
    const Topo t = check_topology(tets_cuda, nbr_cuda, false);
    const std::uint64_t N = static_cast<std::uint64_t>(t.n);
    if (labels.ndim() != 1 || static_cast<std::uint64_t>(labels.shape(0)) != N)
        throw std::runtime_error("labels size mismatch");
    if (N > 0xFFFFFFFFull) throw std::runtime_error(">2^32 full tets unsupported");
    const std::uint64_t nv = static_cast<std::uint64_t>(vertices.shape(0));
    void* stream = current_stream(t.device);
    py::array_t<std::uint8_t> out = label_array(N);
    gpupr_cut_stats st{};
    gpupr_status rc;
    {
        py::gil_scoped_release nogil;
        rc = gpupr_graph_cut(vertices.data(), nv, 0, reinterpret_cast<const std::int32_t*>(t.tets),
                             reinterpret_cast<const std::int32_t*>(t.nbrs), N, labels.data(), 0,
                             fill_T, threads, global_relabel_period, max_rounds, local_steps,
                             out.mutable_data(), 0, stream, &st);
    }
    if (rc != GPUPR_OK) raise_status(rc);
    t_last = st;
    if (N && st.free_n == 0) {
        // bindings.cpp:191-196: the reference's 16-tuple early return
        return py::make_tuple(out, 0, 0, 0, 0, py::int_(st.full_E), 0, py::int_(st.fixed_source),
                              py::int_(st.fixed_sink), 0, py::int_(st.threads), 0, 0, 0, 0.0,
                              py::int_(st.local_steps));
    }
    if (N == 0) {
        return py::make_tuple(out, 0, 0, 0, 0, 0, 0, 0, 0, 0, py::int_(st.threads), 0, 0, 0, 0.0,
                              py::int_(st.local_steps));
    }
    if (verbose()) {
        std::cout << "[GPUPr-B200] build=" << st.build_seconds << "s | free nodes=" << st.free_n
                  << " | solve=" << st.solve_seconds << "s | rounds=" << st.rounds
                  << " | global_relabels=" << st.global_relabels
                  << " | final_relabel=" << st.final_relabel_seconds
                  << "s | flow=" << st.adjusted_flow << std::endl;
    }
    return py::make_tuple(out, py::int_(st.adjusted_flow), py::int_(st.raw_flow),
                          py::int_(st.graph_bytes), py::int_(st.workspace_bytes),
                          py::int_(st.full_E), py::int_(st.free_E), py::int_(st.fixed_source),
                          py::int_(st.fixed_sink), py::int_(st.terminal_edges),
                          py::int_(st.threads), py::int_(st.rounds),
                          py::int_(st.global_relabels), py::int_(st.map_bytes),
                          py::float_(st.build_seconds), py::int_(st.local_steps),
                          py::float_(st.solve_seconds), py::float_(st.native_total_seconds));
}

py::tuple surface_extraction_topology_cuda(U8 labels, F64 vertices, py::object tets_cuda,
                                           py::object nbr_cuda, int threads)
{
    (void)threads;  // the order does not depend on it (bindings.cpp:469-470)
    if (vertices.ndim() != 2 || vertices.shape(1) != 3)
        throw std::runtime_error("vertices must be float64 Nx3");
    const Topo t = check_topology(tets_cuda, nbr_cuda, true);
    const std::uint64_t N = static_cast<std::uint64_t>(t.n);
    if (labels.ndim() != 1 || static_cast<std::uint64_t>(labels.shape(0)) != N)
        throw std::runtime_error("labels size mismatch");
    const std::uint64_t nv = static_cast<std::uint64_t>(vertices.shape(0));
    void* stream = current_stream(t.device);
    std::uint64_t nf = 0, nu = 0;
    gpupr_status rc;
    {
        py::gil_scoped_release nogil;
        rc = gpupr_surface_count(labels.data(), 0, vertices.data(), nv, 0,
                                 reinterpret_cast<const std::int32_t*>(t.tets),
                                 reinterpret_cast<const std::int32_t*>(t.nbrs), N, &nf, &nu, stream);
    }
    if (rc != GPUPR_OK) raise_status(rc);
    py::array_t<double> OV({static_cast<py::ssize_t>(nu), py::ssize_t(3)});
    py::array_t<std::int32_t> OF({static_cast<py::ssize_t>(nf), py::ssize_t(3)});
    {
        py::gil_scoped_release nogil;
        rc = gpupr_surface_fetch(OF.mutable_data(), OV.mutable_data(), 0, stream);
    }
    if (rc != GPUPR_OK) raise_status(rc);
    return py::make_tuple(OV, OF);
}

// wtivo.py:284-309: Nx4 topology (any integer layout numpy accepts) -> one
// contiguous int32 CUDA tensor on the current device, same shape check and
// message; the copy goes through pinned staging with a parallel row gather
// instead of 262k-row host repacks and blocking pageable copies.
py::object topology_to_cuda_chunked(py::object host_array, const std::string& tag)
{
    py::module_ np = py::module_::import("numpy");
    py::array a = np.attr("asarray")(host_array);
    if (a.ndim() != 2 || a.shape(1) != 4)
        throw std::runtime_error(tag + ": expected Nx4 topology array, got " +
                                 std::string(py::str(a.attr("shape"))));
    const char kind = a.dtype().kind();
    const int item = (int)a.itemsize();
    if (!((kind == 'i' || kind == 'u') && (item == 4 || item == 8)))
        a = np.attr("asarray")(a, np.attr("int64"));
    const int eb = (int)a.itemsize();
    const std::uint64_t n = static_cast<std::uint64_t>(a.shape(0));
    py::module_ torch = py::module_::import("torch");
    py::object out = torch.attr("empty")(py::make_tuple(n, 4), py::arg("dtype") = torch.attr("int32"),
                                         py::arg("device") = "cuda");
    const int device = out.attr("device").attr("index").cast<int>();
    void* stream = current_stream(device);
    auto* dst = reinterpret_cast<std::int32_t*>(out.attr("data_ptr")().cast<uintptr_t>());
    const void* src = a.data();
    const std::int64_t rs = a.strides(0), cs = a.strides(1);
    gpupr_status rc;
    {
        py::gil_scoped_release nogil;
        rc = gpupr_upload_topology(src, n, rs, cs, eb, dst, stream);
    }
    if (rc != GPUPR_OK) raise_status(rc);
    return out;
}

// native/core/wtivo_core.cpp:402-464 (is_watertight): same argument check,
// message and 4-tuple (watertight, bad edge groups, seconds, edge buffer
// bytes; the last is this implementation's device edge table).  faces may
// also be a CUDA int32 Fx3 tensor, audited in place.
py::tuple is_watertight(py::object faces, int threads)
{
    (void)threads;
    const auto t0 = std::chrono::steady_clock::now();
    const char* msg = "is_watertight expects Fx3 int32 faces";
    py::module_ torch = py::module_::import("torch");
    const int32_t* ptr = nullptr;
    std::uint64_t nf = 0;
    int on_device = 0;
    void* stream = nullptr;
    py::object keep;
    if (py::isinstance(faces, torch.attr("Tensor")) && faces.attr("is_cuda").cast<bool>()) {
        if (!py::object(faces.attr("dtype")).equal(torch.attr("int32")) ||
            faces.attr("dim")().cast<int64_t>() != 2 || faces.attr("size")(1).cast<int64_t>() != 3 ||
            !faces.attr("is_contiguous")().cast<bool>())
            throw std::runtime_error(msg);
        nf = faces.attr("size")(0).cast<std::uint64_t>();
        ptr = reinterpret_cast<const int32_t*>(faces.attr("data_ptr")().cast<uintptr_t>());
        on_device = 1;
        stream = current_stream(faces.attr("device").attr("index").cast<int>());
        keep = faces;
    } else {
        py::array_t<std::int32_t, py::array::c_style | py::array::forcecast> a =
            py::array_t<std::int32_t, py::array::c_style | py::array::forcecast>::ensure(faces);
        if (!a || a.ndim() != 2 || a.shape(1) != 3) throw std::runtime_error(msg);
        nf = static_cast<std::uint64_t>(a.shape(0));
        ptr = a.data();
        keep = a;
        if (nf) stream = current_stream(torch.attr("cuda").attr("current_device")().cast<int>());
    }
    if (nf == 0) return py::make_tuple(false, py::int_(0), py::float_(0.0), py::int_(0));
    std::uint64_t bad = 0, bytes = 0;
    gpupr_status rc;
    {
        py::gil_scoped_release nogil;
        rc = gpupr_edge_audit(ptr, nf, on_device, &bad, &bytes, stream);
    }
    if (rc != GPUPR_OK) raise_status(rc);
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (verbose())
        std::cout << "[WTiVo-Watertight] faces=" << nf << " | bad-edge-groups=" << bad
                  << " | total=" << sec << "s" << std::endl;
    return py::make_tuple(py::bool_(bad == 0), py::int_(bad), py::float_(sec), py::int_(bytes));
}

// The UDF side of native/vdb/wtivo_vdb.cpp's SparseUDF, for the label query
// only: a brick grid (8^3-voxel bricks, a dense brick table, a background)
// held in device memory as torch tensors, and sample_tet_labels with the
// reference method's arguments, checks, messages and (labels, seconds)
// return (wtivo_vdb.cpp:1519-1584).
class BrickUDF {
public:
    BrickUDF(py::object values, py::object table, py::object origin, double voxel_size,
             float background)
        : voxel_size_(voxel_size), background_(background)
    {
        if (!(voxel_size > 0.0)) throw std::runtime_error("BrickUDF: voxel_size must be > 0");
        py::module_ np = py::module_::import("numpy");
        py::module_ torch = py::module_::import("torch");
        py::array_t<std::int32_t, py::array::c_style | py::array::forcecast> tab =
            py::array_t<std::int32_t, py::array::c_style | py::array::forcecast>::ensure(table);
        py::array_t<float, py::array::c_style | py::array::forcecast> val =
            py::array_t<float, py::array::c_style | py::array::forcecast>::ensure(values);
        py::array_t<std::int64_t, py::array::c_style | py::array::forcecast> org =
            py::array_t<std::int64_t, py::array::c_style | py::array::forcecast>::ensure(origin);
        if (!tab || tab.ndim() != 3) throw std::runtime_error("BrickUDF: table must be int32 [bx, by, bz]");
        if (!val || val.size() % 512 != 0) throw std::runtime_error("BrickUDF: values must be float32 [bricks, 8, 8, 8]");
        if (!org || org.size() != 3) throw std::runtime_error("BrickUDF: origin must have length 3");
        for (int k = 0; k < 3; ++k) {
            dims_[k] = (int32_t)tab.shape(k);
            origin_[k] = (int32_t)org.data()[k];
        }
        n_bricks_ = (std::uint64_t)(val.size() / 512);
        const std::int32_t* tp = tab.data();
        for (py::ssize_t i = 0; i < tab.size(); ++i)
            if (tp[i] < -1 || (tp[i] >= 0 && (std::uint64_t)tp[i] >= n_bricks_))
                throw std::runtime_error("BrickUDF: table entry out of range");
        table_ = torch.attr("from_numpy")(tab.attr("reshape")(-1)).attr("cuda")();
        values_ = torch.attr("from_numpy")(val.attr("reshape")(-1)).attr("cuda")();
    }

    py::tuple sample_tet_labels(py::object tet_vertices, py::object tets, py::object bbox_min,
                                py::object bbox_max, double padding, double threshold, int threads)
    {
        (void)threads;
        const std::string pre = "SparseUDF.sample_tet_labels: ";
        py::module_ torch = py::module_::import("torch");
        F64 V = F64::ensure(tet_vertices);
        if (!V || V.ndim() != 2 || V.shape(1) != 3)
            throw std::runtime_error(pre + "tet_vertices must be float64 Nx3");
        const int32_t* tp = nullptr;
        std::uint64_t nt = 0;
        int t_dev = 0;
        py::object keep;
        if (py::isinstance(tets, torch.attr("Tensor")) && tets.attr("is_cuda").cast<bool>()) {
            if (!py::object(tets.attr("dtype")).equal(torch.attr("int32")) || tets.attr("dim")().cast<int64_t>() != 2 ||
                tets.attr("size")(1).cast<int64_t>() != 4 || !tets.attr("is_contiguous")().cast<bool>())
                throw std::runtime_error(pre + "tets must be int32 Mx4");
            nt = tets.attr("size")(0).cast<std::uint64_t>();
            tp = reinterpret_cast<const int32_t*>(tets.attr("data_ptr")().cast<uintptr_t>());
            t_dev = 1;
            keep = tets;
        } else {
            py::array_t<std::int32_t, py::array::c_style | py::array::forcecast> T =
                py::array_t<std::int32_t, py::array::c_style | py::array::forcecast>::ensure(tets);
            if (!T || T.ndim() != 2 || T.shape(1) != 4) throw std::runtime_error(pre + "tets must be int32 Mx4");
            nt = (std::uint64_t)T.shape(0);
            tp = T.data();
            keep = T;
        }
        F64 bmin = F64::ensure(bbox_min), bmax = F64::ensure(bbox_max);
        if (!bmin || !bmax || bmin.ndim() != 1 || bmin.shape(0) != 3 || bmax.ndim() != 1 || bmax.shape(0) != 3)
            throw std::runtime_error(pre + "bbox must have length 3");
        py::array_t<std::uint8_t> labels(static_cast<py::ssize_t>(nt));
        gpupr_brick_grid g{};
        g.voxel_size = voxel_size_;
        for (int k = 0; k < 3; ++k) {
            g.origin[k] = origin_[k];
            g.dims[k] = dims_[k];
        }
        g.background = background_;
        g.on_device = 1;
        g.table = reinterpret_cast<const int32_t*>(table_.attr("data_ptr")().cast<uintptr_t>());
        g.values = reinterpret_cast<const float*>(values_.attr("data_ptr")().cast<uintptr_t>());
        g.n_bricks = n_bricks_;
        void* stream = current_stream(table_.attr("device").attr("index").cast<int>());
        const double* vp = V.data();
        const std::uint64_t nv = (std::uint64_t)V.shape(0);
        const double* b0 = bmin.data();
        const double* b1 = bmax.data();
        std::uint8_t* lp = labels.mutable_data();
        const auto t0 = std::chrono::steady_clock::now();
        gpupr_status rc;
        {
            py::gil_scoped_release nogil;
            rc = gpupr_sample_tet_labels(&g, vp, nv, 0, tp, nt, t_dev, b0, b1, padding, threshold, lp, 0,
                                         nullptr, stream);
        }
        if (rc != GPUPR_OK) raise_status(rc);
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return py::make_tuple(labels, sec);
    }

    py::dict stats() const
    {
        py::dict d;
        d["voxel_size"] = voxel_size_;
        d["background"] = background_;
        d["bricks"] = n_bricks_;
        d["dims"] = py::make_tuple(dims_[0], dims_[1], dims_[2]);
        d["origin"] = py::make_tuple(origin_[0], origin_[1], origin_[2]);
        d["device_bytes"] = (std::uint64_t)(n_bricks_ * 2048u + (std::uint64_t)dims_[0] * dims_[1] * dims_[2] * 4u);
        return d;
    }

private:
    double voxel_size_;
    float background_;
    int32_t origin_[3] = {0, 0, 0}, dims_[3] = {0, 0, 0};
    std::uint64_t n_bricks_ = 0;
    py::object table_, values_;
};

py::dict last_stats()
{
    const gpupr_cut_stats& s = t_last;
    py::dict d;
    d["adjusted_flow"] = s.adjusted_flow;
    d["raw_flow"] = s.raw_flow;
    d["graph_bytes"] = s.graph_bytes;
    d["workspace_bytes"] = s.workspace_bytes;
    d["free_n"] = s.free_n;
    d["n_full"] = s.n_full;
    d["rounds"] = s.rounds;
    d["global_relabels"] = s.global_relabels;
    d["build_seconds"] = s.build_seconds;
    d["solve_seconds"] = s.solve_seconds;
    d["final_relabel_seconds"] = s.final_relabel_seconds;
    d["partition_seconds"] = s.partition_seconds;
    d["native_total_seconds"] = s.native_total_seconds;
    d["node_visits"] = s.node_visits;
    d["pushes"] = s.pushes;
    d["bfs_visits"] = s.bfs_visits;
    d["bfs_levels"] = s.bfs_levels;
    d["kernel_launches"] = s.kernel_launches;
    d["solve_device_ms"] = s.solve_device_ms;
    d["build_device_ms"] = s.build_device_ms;
    return d;
}

}  // namespace

PYBIND11_MODULE(wtivo_gpupr, m)
{
    m.doc() = "WTiVo graph cut on B200: GPU reduced-graph build, multi-discharge push-relabel "
              "with exact global relabels, and GPU cut-surface extraction";
    m.def("graph_cut_fast", &graph_cut_fast, py::arg("vertices"), py::arg("tets_cuda"),
          py::arg("neighbors_cuda"), py::arg("labels"), py::arg("fill_T"), py::arg("threads") = 16,
          py::arg("global_relabel_period") = 1024, py::arg("max_rounds") = 2000000ULL,
          py::arg("local_steps") = 8);
    m.def("graph_cut_gpupr_fast_v630", &graph_cut_fast, py::arg("vertices"), py::arg("tets_cuda"),
          py::arg("neighbors_cuda"), py::arg("labels"), py::arg("fill_T"), py::arg("threads") = 16,
          py::arg("global_relabel_period") = 1024, py::arg("max_rounds") = 2000000ULL,
          py::arg("local_steps") = 8);
    m.def("surface_extraction_topology_cuda", &surface_extraction_topology_cuda, py::arg("labels"),
          py::arg("vertices"), py::arg("tets_cuda"), py::arg("neighbors_cuda"),
          py::arg("threads") = 16);
    py::class_<BrickUDF>(m, "BrickUDF",
                         "Sparse unsigned distance grid (8^3-voxel bricks) on the GPU for the "
                         "tet-centroid label query (replaces SparseUDF.sample_tet_labels).")
        .def(py::init<py::object, py::object, py::object, double, float>(), py::arg("values"),
             py::arg("table"), py::arg("origin"), py::arg("voxel_size"), py::arg("background"))
        .def("sample_tet_labels", &BrickUDF::sample_tet_labels, py::arg("tet_vertices"), py::arg("tets"),
             py::arg("bbox_min"), py::arg("bbox_max"), py::arg("padding"), py::arg("threshold"),
             py::arg("threads") = 16)
        .def("stats", &BrickUDF::stats);
    m.def("is_watertight", &is_watertight, py::arg("faces"), py::arg("threads") = 0,
          "Edge-degree watertight audit on the GPU (replaces wtivo_core.is_watertight).");
    m.def("topology_to_cuda_chunked", &topology_to_cuda_chunked, py::arg("host_array"),
          py::arg("tag") = "topology",
          "Nx4 host topology -> contiguous int32 CUDA tensor (replaces wtivo.py's helper).");
    m.def("last_stats", &last_stats,
          "Extended statistics of the last graph_cut_fast call on this thread.");
    m.def("release_cached_memory", []() {
        const gpupr_status rc = gpupr_release_cached_memory();
        if (rc != GPUPR_OK) raise_status(rc);
    });
    m.attr("abi_version") = gpupr_abi_version();
}
