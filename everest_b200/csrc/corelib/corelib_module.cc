// pybind11 module `corelib` with submodule `data`: the names
// system/tmine/core.py imports from the reference's module
// (src/mods/corelib.cc:17-190).  run() releases the GIL.
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>
#include <pybind11/stl/filesystem.h>
#include <pybind11/stl_bind.h>

#include <cstring>
#include <sstream>

#include "corelib.h"

namespace py = pybind11;
using namespace corelib;

PYBIND11_MAKE_OPAQUE(corelib::data::HostGraphDataList);
PYBIND11_MAKE_OPAQUE(corelib::data::SubPartitionList);

PYBIND11_MODULE(corelib, m) {
  m.doc() = "B200 temporal-motif miner: the reference's corelib API over sm_100a kernels";
  auto d = m.def_submodule("data");
  py::bind_vector<data::HostGraphDataList>(d, "HostGraphDataList");
  py::bind_vector<data::SubPartitionList>(d, "SubPartitionList");

  py::class_<data::EdgeListLoader>(d, "EdgeListLoader", "A dataloader that loads edge list")
      .def(py::init<std::filesystem::path, bool>(), py::arg("pathToGraph"), py::arg("useCache") = true)
      .def("name", &data::EdgeListLoader::name)
      .def("edgeListLength", &data::EdgeListLoader::edgeListLength)
      .def("__repr__", [](const data::EdgeListLoader &e) { return "EdgeListLoader Object <" + e.name() + ">"; });

  py::class_<data::FeatureLoader>(d, "FeatureLoader", "Random features (optional on this path)")
      .def(py::init<const data::EdgeListLoader *, std::filesystem::path>(), py::keep_alive<1, 2>())
      .def("name", &data::FeatureLoader::name)
      .def("edgeFeaturesLength", &data::FeatureLoader::edgeFeaturesLength)
      .def("verticesFeaturesLength", &data::FeatureLoader::verticesFeaturesLength)
      .def("__repr__", [](const data::FeatureLoader &e) { return "FeatureLoader Object <" + e.name() + ">"; });

  py::class_<data::HostGraphData>(d, "HostGraphData", "The graph data for a subset of edge list")
      .def_readonly("name", &data::HostGraphData::name)
      .def_readonly("beg", &data::HostGraphData::beg)
      .def_readonly("end", &data::HostGraphData::end)
      .def_readonly("numEdges", &data::HostGraphData::numEdges)
      .def_readonly("numVertices", &data::HostGraphData::numVertices)
      .def_readonly("totalBytes", &data::HostGraphData::totalBytes)
      .def_readonly("Eg", &data::HostGraphData::Eg)
      .def_readonly("edgeFeatures", &data::HostGraphData::edgeFeatures)
      .def_readonly("verticesFeatures", &data::HostGraphData::verticesFeatures)
      .def("__repr__", [](const data::HostGraphData &e) {
        std::ostringstream s;
        s << "<HostGraphData>\nname: " << e.name << "\nbeg: " << e.beg << ", end: " << e.end
          << "\nnumEdges: " << e.numEdges << ", numVertices: " << e.numVertices
          << ", totalBytes: " << e.totalBytes;
        return s.str();
      });

  py::class_<data::SubPartition>(d, "SubPartition", "A sub-partition of edge list")
      .def_readwrite("beg", &data::SubPartition::beg)
      .def_readwrite("end", &data::SubPartition::end)
      .def_readwrite("n", &data::SubPartition::n)
      .def("__repr__", [](const data::SubPartition &e) {
        return "<SubPartition: " + std::to_string(e.beg) + " " + std::to_string(e.end) + " " +
               std::to_string(e.n) + ">";
      });

  d.def("divideList", &data::divideList);
  d.def("removeMinor", &data::removeMinor);
  d.def("includeMinor", &data::includeMinor);

  py::class_<data::GraphDataLoader>(d, "GraphDataLoader", "A dataloader that loads graph data")
      .def(py::init<const data::EdgeListLoader *, const data::FeatureLoader *>(), py::keep_alive<1, 2>(),
           py::keep_alive<1, 3>())
      .def("createGraphData", &data::GraphDataLoader::createGraphData, py::arg("beg") = 0,
           py::arg("end") = 0, py::arg("cache") = true)
      .def("createPartitionsData", &data::GraphDataLoader::createPartitionsData)
      .def("createPartitionsDataMajor", &data::GraphDataLoader::createPartitionsDataMajor)
      .def("createPartitionsDataMinor", &data::GraphDataLoader::createPartitionsDataMinor)
      .def("__repr__", [](const data::GraphDataLoader &e) { return "<GraphDataLoader: " + e.name() + ">"; });

  py::class_<data::DeviceGraphData>(d, "DeviceGraphData", "The graph data on a device")
      .def_readonly("device", &data::DeviceGraphData::device)
      .def_readonly("numEdges", &data::DeviceGraphData::numEdges)
      .def_readonly("numVertices", &data::DeviceGraphData::numVertices)
      .def("__repr__", [](const data::DeviceGraphData &e) {
        return "<DeviceGraphData: device " + std::to_string(e.device) + ", " + std::to_string(e.numEdges) +
               " edges>";
      });

  py::class_<data::GraphDataManager>(d, "GraphDataManager", "Moves host graphs to devices")
      .def("allocBatch", &data::GraphDataManager::allocBatch)
      .def("alloc", &data::GraphDataManager::alloc)
      .def("moveAsync", &data::GraphDataManager::moveAsync, py::call_guard<py::gil_scoped_release>())
      .def("waitMove", &data::GraphDataManager::waitMove)
      .def("__repr__", [](const data::GraphDataManager &) { return std::string("<GraphDataManager>"); });
  d.def("MakeGraphDataManager", &data::MakeGraphDataManager);

  py::class_<data::HostMotifData>(d, "HostMotifData", "Motif Data on the host")
      .def(py::init<const std::filesystem::path &>())
      .def_static("fromText", &data::HostMotifData::fromText, py::arg("text"), py::arg("name") = "motif")
      .def_readonly("name", &data::HostMotifData::name)
      .def_readonly("numEdges", &data::HostMotifData::numEdges)
      .def_readonly("numVertices", &data::HostMotifData::numVertices)
      .def("motifEdges",
           [](const data::HostMotifData &m) {
             std::vector<int> mu, mv;
             for (auto &e : m.edges) {
               mu.push_back(e.u);
               mv.push_back(e.v);
             }
             return std::make_pair(mu, mv);
           },
           "(sources, targets) of the relabeled motif edges")
      .def_property_readonly("edges", [](const data::HostMotifData &e) {
        std::vector<std::tuple<int, int, int>> r;
        for (auto &x : e.edges) r.emplace_back(x.u, x.v, x.t);
        return r;
      })
      .def_property_readonly("minfo", [](const data::HostMotifData &e) {
        std::vector<std::tuple<int, int, int, int, bool>> r;
        for (auto &x : e.minfo) r.emplace_back(x.baseNode, x.constraintNode, x.mappedNodes, x.io, x.newNode);
        return r;
      })
      .def("__repr__", [](const data::HostMotifData &e) {
        std::ostringstream s;
        s << "<HostMotifData>\nname: " << e.name << ", numEdges: " << e.numEdges
          << ", numVertices: " << e.numVertices << "\nEdges:";
        for (auto &x : e.edges) s << "\n" << x.u << " " << x.v << " " << x.t;
        return s.str();
      });

  py::class_<data::DeviceJobData>(d, "DeviceJobData", "Job Data on the Device")
      .def(py::init<const data::DeviceGraphData &, const data::HostMotifData &>())
      .def("__repr__", [](const data::DeviceJobData &e) {
        return "<DeviceJobData: device " + std::to_string(e.device) + ", motif edges " +
               std::to_string(e.motifNumEdges) + ">";
      });

  py::class_<data::MineJob>(d, "MineJob", "A Job, contains everything to let a worker to mine")
      .def(py::init<const data::DeviceJobData *, int, int, int>(), py::arg("_data"), py::arg("_delta"),
           py::arg("_beg") = 0, py::arg("_end") = -1, py::keep_alive<1, 2>())
      .def("getWork", &data::MineJob::getWork)
      .def("setWork", &data::MineJob::setWork)
      .def("__repr__", [](const data::MineJob &e) {
        return "<MineJob: " + std::to_string(e.device) + ", " + std::to_string(e.delta) + ", " +
               std::to_string(e.beg) + ", " + std::to_string(e.end) + ">";
      });

  py::class_<GPUWorker>(m, "GPUWorker", "GPU worker class")
      .def("run", &GPUWorker::run, py::call_guard<py::gil_scoped_release>())
      .def("take", &GPUWorker::take, py::keep_alive<1, 2>())
      .def("update_job", &GPUWorker::update_job)
      .def("timed_run", &GPUWorker::timed_run, py::call_guard<py::gil_scoped_release>())
      .def("time", &GPUWorker::time)
      .def("count", &GPUWorker::count)
      .def("clear_time", &GPUWorker::clear_time)
      .def("pause", &GPUWorker::pause)
      .def("printEnum", &GPUWorker::printEnum)
      .def("configure", &GPUWorker::configure, py::arg("enumCap"), py::arg("flags") = 0u)
      .def(
          "setConstraints",
          [](GPUWorker &w, py::object blob) {
            if (blob.is_none()) {
              w.setConstraints(nullptr);
              return;
            }
            const std::string s = blob.cast<py::bytes>();
            if (s.size() != sizeof(evx_constraints))
              throw std::invalid_argument("setConstraints: expected the " + std::to_string(sizeof(evx_constraints)) +
                                          "-byte evx_constraints struct");
            evx_constraints c;
            std::memcpy(&c, s.data(), sizeof(c));
            w.setConstraints(&c);
          },
          py::arg("constraints"),
          "bytes of an evx_constraints struct (everest_b200.constraints), or None")
      .def("setTuning", &GPUWorker::setTuning)
      .def("lastDeviceMs", &GPUWorker::lastDeviceMs)
      .def("lastKernelLaunches", &GPUWorker::lastKernelLaunches)
      .def("__repr__", [](const GPUWorker &w) {
        return "<GPUWorker>\ntype: " + w.type_ + ", gpu: " + std::to_string(w.gpu_) +
               ", count: " + std::to_string(w.count_) + ", time: " + std::to_string(w.time_);
      });

  py::class_<GPUWorkerLibManager>(m, "GPUWorkerLibManager", "to manage GPU worker libraries")
      .def(py::init<>())
      .def("openLib", &GPUWorkerLibManager::openLib)
      .def("unloadLib", &GPUWorkerLibManager::unloadLib)
      .def("construct", &GPUWorkerLibManager::construct)
      .def("__repr__", [](const GPUWorkerLibManager &e) { return "<GPUWorkerLibManager>\n" + e.toString(); });

  auto single = [&](auto &cls) {
    using C = typename std::remove_reference_t<decltype(cls)>::type;
    cls.def("setHostGraph", &C::setHostGraph, py::arg("hostGraph"), py::arg("n") = -1,
            py::keep_alive<1, 2>(), py::call_guard<py::gil_scoped_release>())
        .def("setHostMotif", &C::setHostMotif, py::keep_alive<1, 2>())
        .def("setWorker", &C::setWorker, py::keep_alive<1, 2>())
        .def("run", &C::run, py::call_guard<py::gil_scoped_release>())
        .def("__repr__", [](const C &) { return std::string("<SingleGPUExeuction>"); });
  };
  py::class_<SingleGPUExecution> s1(m, "SingleGPUExecution", "SingleGPUExecution uses a single GPU to do the mining");
  s1.def(py::init<const data::GraphDataManager *, int>(), py::arg("dataManager"), py::arg("device") = 0,
         py::keep_alive<1, 2>());
  single(s1);
  py::class_<SingleGPUExecutionDiv> s2(m, "SingleGPUExecutionDiv", "Splits the roots into div jobs on one GPU");
  s2.def(py::init<const data::GraphDataManager *, int, int>(), py::arg("dataManager"), py::arg("device") = 0,
         py::arg("div") = 64, py::keep_alive<1, 2>());
  single(s2);
  py::class_<SingleGPUExecutionPause> s3(m, "SingleGPUExecutionPause", "Runs to completion (pause is reserved)");
  s3.def(py::init<const data::GraphDataManager *, int>(), py::arg("dataManager"), py::arg("device") = 0,
         py::keep_alive<1, 2>());
  single(s3);

  m.def("SingleGPURunBatch", &SingleGPURunBatch, py::call_guard<py::gil_scoped_release>());

  auto multi = [&](auto &cls, const char *nm) {
    using C = typename std::remove_reference_t<decltype(cls)>::type;
    cls.def(py::init<const data::GraphDataManager *, int>(), py::keep_alive<1, 2>())
        .def("setHostGraphs", &C::setHostGraphs, py::keep_alive<1, 2>())
        .def("setHostMotif", &C::setHostMotif, py::keep_alive<1, 2>())
        .def("setWorkers", &C::setWorkers)
        .def("run", &C::run, py::call_guard<py::gil_scoped_release>())
        .def("numDevice", &C::numDevice)
        .def("__repr__", [nm](const C &e) { return std::string("<") + nm + ": " + std::to_string(e.numDevice()) + ">"; });
  };
  py::class_<MultiGPUExecutionNaive> m1(m, "MultiGPUExecutionNaive", "One device only on this path");
  multi(m1, "MultiGPUExecutionNaive");
  py::class_<MultiGPUExecutionDyn> m2(m, "MultiGPUExecutionDyn", "One device only on this path");
  multi(m2, "MultiGPUExecutionDyn");
  py::class_<MultiGPUExecutionDynPause> m3(m, "MultiGPUExecutionDynPause", "One device only on this path");
  multi(m3, "MultiGPUExecutionDynPause");

  m.def("allCount", &allCount);
  m.attr("FLAG_STRICT_TS") = (unsigned)EVX_FLAG_STRICT_TS;
  m.attr("FLAG_EXACT_TOTAL") = (unsigned)EVX_FLAG_EXACT_TOTAL;
  m.attr("FLAG_NO_STEAL") = (unsigned)EVX_FLAG_NO_STEAL;
}
