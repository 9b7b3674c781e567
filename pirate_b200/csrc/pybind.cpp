// pybind.cpp -- the pybind11 module pirate_b200._pirate_b200_pybind: pirate's pybind11 classes
// (src_pybind11/pirate_pybind11.cpp:453-593) over the C++ classes of include/pirate_b200.hpp.
//
// Names and argument conventions follow pirate's module: DedispersionConfig.from_yaml,
// DedispersionPlan(config) with .trees, GpuDedisperser(plan, cuda_device_id, num_consumers, ...)
// with allocate(), _acquire_input(seq_id, stream_ptr), _release_input_and_launch_dd_kernels(seq_id,
// stream_ptr), _acquire_output(consumer_id, seq_id, stream_ptr), _release_output(consumer_id, seq_id,
// stream_ptr), fill_all_weights, fill_analytic_weights. As in pirate, the four seq_id calls and
// allocate release the GIL, so producer and consumer threads run concurrently. Device arrays are
// returned as (pointer, shape) pairs; pirate_b200/__init__.py wraps them as torch tensors.

#include "../../include/pirate_b200.hpp"

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

namespace py = pybind11;
using namespace pirate_b200;

PYBIND11_MODULE(_pirate_b200_pybind, m)
{
    m.doc() = "pybind11 surface of pirate_b200 (pirate's DedispersionConfig / DedispersionPlan / GpuDedisperser)";

    py::class_<DedispersionConfig>(m, "DedispersionConfig")
        .def_static("from_yaml", &DedispersionConfig::from_yaml, py::arg("filename"))
        .def_static("from_yaml_string", &DedispersionConfig::from_yaml_string, py::arg("text"))
        .def("to_yaml_string", &DedispersionConfig::to_yaml_string)
        .def("dm_per_unit_delay", &DedispersionConfig::dm_per_unit_delay);

    py::class_<pb2_tree_info>(m, "DedispersionTree")
        .def_readonly("primary_tree_index", &pb2_tree_info::primary_tree_index)
        .def_readonly("early_trigger_level", &pb2_tree_info::early_trigger_level)
        .def_readonly("amb_rank", &pb2_tree_info::amb_rank)
        .def_readonly("dd_rank", &pb2_tree_info::dd_rank)
        .def_readonly("nt_ds", &pb2_tree_info::nt_ds)
        .def_readonly("ndm_out", &pb2_tree_info::ndm_out)
        .def_readonly("nt_out", &pb2_tree_info::nt_out)
        .def_readonly("ndm_wt", &pb2_tree_info::ndm_wt)
        .def_readonly("nt_wt", &pb2_tree_info::nt_wt)
        .def_readonly("nprofiles", &pb2_tree_info::nprofiles)
        .def_readonly("Dcore", &pb2_tree_info::Dcore)
        .def_readonly("nsubbands", &pb2_tree_info::nsubbands)
        .def_readonly("nmultiplets", &pb2_tree_info::nmultiplets)
        .def_readonly("pf_rank", &pb2_tree_info::pf_rank)
        .def_readonly("dm_min", &pb2_tree_info::dm_min)
        .def_readonly("dm_max", &pb2_tree_info::dm_max);

    py::class_<DedispersionPlan, std::shared_ptr<DedispersionPlan>>(m, "DedispersionPlan")
        .def(py::init<const DedispersionConfig &>(), py::arg("config"))
        .def_readonly("ntrees", &DedispersionPlan::ntrees)
        .def_readonly("trees", &DedispersionPlan::trees)
        .def("decode_argmax", [](const DedispersionPlan &p, uint32_t token, long itree, long idm, long itime) {
                long fmin, fmax, tlo, thi, pp;
                p.decode_argmax(token, itree, idm, itime, fmin, fmax, tlo, thi, pp);
                return py::make_tuple(fmin, fmax, tlo, thi, pp);
            }, py::arg("token"), py::arg("itree"), py::arg("idm"), py::arg("itime"));

    py::class_<GpuDedisperser::Outputs>(m, "Outputs")
        .def_readonly("dtype", &GpuDedisperser::Outputs::dtype)
        .def_readonly("nbeams", &GpuDedisperser::Outputs::nbeams)
        .def_readonly("ichunk_zero_based", &GpuDedisperser::Outputs::ichunk_zero_based)
        .def_readonly("ichunk_fpga_based", &GpuDedisperser::Outputs::ichunk_fpga_based)
        .def_readonly("ibeam", &GpuDedisperser::Outputs::ibeam)
        .def_readonly("ndm_out", &GpuDedisperser::Outputs::ndm_out)
        .def_readonly("nt_out", &GpuDedisperser::Outputs::nt_out)
        .def_property_readonly("out_max_ptrs", [](const GpuDedisperser::Outputs &o) {
                std::vector<uintptr_t> v;
                for (void *p : o.out_max) v.push_back(reinterpret_cast<uintptr_t>(p));
                return v;
            })
        .def_property_readonly("out_argmax_ptrs", [](const GpuDedisperser::Outputs &o) {
                std::vector<uintptr_t> v;
                for (uint32_t *p : o.out_argmax) v.push_back(reinterpret_cast<uintptr_t>(p));
                return v;
            });

    py::class_<GpuDedisperser, std::shared_ptr<GpuDedisperser>>(m, "GpuDedisperser")
        .def(py::init([](std::shared_ptr<DedispersionPlan> plan, int cuda_device_id, long num_consumers, long nbatches_out,
                         long nbatches_wt, long initial_chunk, bool synchronous, long release_timeout_ms) {
                GpuDedisperser::Params p;
                p.cuda_device_id = cuda_device_id;
                p.num_consumers = num_consumers;
                p.nbatches_out = nbatches_out;
                p.nbatches_wt = nbatches_wt;
                p.initial_chunk = initial_chunk;
                p.synchronous = synchronous;
                p.release_timeout_ms = release_timeout_ms;
                return GpuDedisperser::create(*plan, p);
            }),
            py::arg("plan"), py::arg("cuda_device_id") = 0, py::arg("num_consumers") = 1, py::arg("nbatches_out") = 0,
            py::arg("nbatches_wt") = 0, py::arg("initial_chunk") = 0, py::arg("synchronous") = false,
            py::arg("release_timeout_ms") = 0)
        .def("allocate", &GpuDedisperser::allocate, py::call_guard<py::gil_scoped_release>())
        .def("device_bytes", &GpuDedisperser::device_bytes)
        .def("_acquire_input", [](GpuDedisperser &d, long seq_id, uintptr_t stream_ptr) {
                long shape[3];
                void *p;
                {
                    py::gil_scoped_release nogil;
                    p = d.acquire_input(seq_id, reinterpret_cast<void *>(stream_ptr), shape);
                }
                return py::make_tuple(reinterpret_cast<uintptr_t>(p), py::make_tuple(shape[0], shape[1], shape[2]));
            }, py::arg("seq_id"), py::arg("stream_ptr"))
        .def("_release_input_and_launch_dd_kernels", [](GpuDedisperser &d, long seq_id, uintptr_t stream_ptr) {
                d.release_input_and_launch_dd_kernels(seq_id, reinterpret_cast<void *>(stream_ptr));
            }, py::arg("seq_id"), py::arg("stream_ptr"), py::call_guard<py::gil_scoped_release>())
        .def("_acquire_output", [](GpuDedisperser &d, long consumer_id, long seq_id, uintptr_t stream_ptr, bool sync) {
                return d.acquire_output(consumer_id, seq_id, reinterpret_cast<void *>(stream_ptr), sync);
            }, py::arg("consumer_id"), py::arg("seq_id"), py::arg("stream_ptr"), py::arg("sync") = false,
            py::call_guard<py::gil_scoped_release>())
        .def("_release_output", [](GpuDedisperser &d, long consumer_id, long seq_id, uintptr_t stream_ptr) {
                d.release_output(consumer_id, seq_id, reinterpret_cast<void *>(stream_ptr));
            }, py::arg("consumer_id"), py::arg("seq_id"), py::arg("stream_ptr"), py::call_guard<py::gil_scoped_release>())
        .def("fill_all_weights", [](GpuDedisperser &d, long itree, py::array_t<float, py::array::c_style | py::array::forcecast> w) {
                const float *p = w.data();
                long n = long(w.size());
                py::gil_scoped_release nogil;
                d.fill_all_weights(itree, p, n);
            }, py::arg("itree"), py::arg("pf_weights"))
        .def("fill_analytic_weights", [](GpuDedisperser &d, py::array_t<double, py::array::c_style | py::array::forcecast> fv) {
                std::vector<double> v(fv.data(), fv.data() + fv.size());
                py::gil_scoped_release nogil;
                d.fill_analytic_weights(v);
            }, py::arg("freq_variances"))
        .def("time", &GpuDedisperser::time, py::arg("niterations"), py::call_guard<py::gil_scoped_release>())
        .def("stop", &GpuDedisperser::stop);
}
