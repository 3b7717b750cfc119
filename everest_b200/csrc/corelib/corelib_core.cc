// corelib implementation over the C ABI.  See corelib.h.
#include "corelib.h"

#include <dlfcn.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace corelib {

#define COREL_API __attribute__((visibility("default")))

std::string check_evx(int rc, const char *what) {
  if (rc == EVX_OK) return {};
  std::string msg = std::string(what) + ": " + evx_last_error();
  if (rc == EVX_ERR_INVALID || rc == EVX_ERR_OVERFLOW) throw std::invalid_argument(msg);
  if (rc == EVX_ERR_IO) throw std::ios_base::failure(msg);
  throw std::runtime_error(msg);
}

namespace {

std::vector<int> take_ints(int *p, size_t n) {
  std::vector<int> v(p, p + n);
  evx_free(p);
  return v;
}

// The first min(n, file length) int32 values of a raw file (a random-feature
// file can be far longer than the graph needs: read only the prefix).
bool read_ints_prefix(const std::filesystem::path &p, size_t n, std::vector<int> &out) {
  std::ifstream f(p, std::ios::binary | std::ios::ate);
  if (!f) return false;
  const std::streamsize sz = f.tellg();
  if (sz < 0) return false;
  const size_t have = (size_t)sz / 4;
  out.resize(std::min(n, have));
  f.seekg(0);
  return (bool)f.read(reinterpret_cast<char *>(out.data()), (std::streamsize)(out.size() * 4));
}

bool read_ints(const std::filesystem::path &p, std::vector<int> &out) {
  std::ifstream f(p, std::ios::binary | std::ios::ate);
  if (!f) return false;
  const std::streamsize sz = f.tellg();
  if (sz < 0 || sz % 4) return false;
  out.resize((size_t)sz / 4);
  f.seekg(0);
  return (bool)f.read(reinterpret_cast<char *>(out.data()), sz);
}

void write_ints(const std::filesystem::path &p, const std::vector<int> &v) {
  std::ofstream f(p, std::ios::binary | std::ios::trunc);
  if (!f) throw std::runtime_error("cannot write cache file " + p.string());
  f.write(reinterpret_cast<const char *>(v.data()), (std::streamsize)(v.size() * sizeof(int)));
}

size_t calc_total_bytes(size_t E, size_t V) {
  // src/core/gpu/data.cu:22-24
  return (sizeof(TemporalEdge) + sizeof(int) * 3) * E + (sizeof(int) * 2) * (V + 1) + sizeof(int) * V;
}

}  // namespace

namespace data {

CacheDirectoryAccess::CacheDirectoryAccess(const std::filesystem::path &pathToGraph, bool create)
    : name_(pathToGraph.stem().string()), graphPath_(pathToGraph),
      cacheDir_(pathToGraph.parent_path() / pathToGraph.stem()) {
  if (create && !std::filesystem::exists(cacheDir_)) {
    std::error_code ec;
    std::filesystem::create_directories(cacheDir_, ec);
  }
}

std::filesystem::path CacheDirectoryAccess::cacheGraphDirPath(size_t beg, size_t end) const {
  return cacheDir_ / (name_ + "-" + std::to_string(beg) + "-" + std::to_string(end));
}

EdgeListLoader::EdgeListLoader(const std::filesystem::path &pathToGraph, bool useCache)
    : CacheDirectoryAccess(pathToGraph, useCache) {
  if (useCache && std::filesystem::exists(cacheUPath()) && std::filesystem::exists(cacheVPath()) &&
      std::filesystem::exists(cacheTPath()) && std::filesystem::exists(cacheIDSPath())) {
    if (read_ints(cacheUPath(), U_) && read_ints(cacheVPath(), V_) && read_ints(cacheTPath(), T_) &&
        read_ints(cacheIDSPath(), IDS_) && U_.size() == V_.size() && U_.size() == T_.size() &&
        U_.size() == IDS_.size())
      return;
  }
  int64_t n = 0;
  int *u = nullptr, *v = nullptr, *t = nullptr, *ids = nullptr;
  check_evx(evx_edgelist_parse(pathToGraph.string().c_str(), &n, &u, &v, &t, &ids),
            "EdgeListLoader");
  U_ = take_ints(u, (size_t)n);
  V_ = take_ints(v, (size_t)n);
  T_ = take_ints(t, (size_t)n);
  IDS_ = take_ints(ids, (size_t)n);
  if (useCache && std::filesystem::exists(cacheDir_)) {
    write_ints(cacheUPath(), U_);
    write_ints(cacheVPath(), V_);
    write_ints(cacheTPath(), T_);
    write_ints(cacheIDSPath(), IDS_);
  }
}

FeatureLoader::FeatureLoader(const EdgeListLoader *eloader, const std::filesystem::path &pathToRands)
    : CacheDirectoryAccess(eloader->graphPath_, false) {
  const size_t E = eloader->edgeListLength();
  // the reference's feature caches (src/core/cpu/data.cc:316-327)
  std::vector<int> fe, fvv, fvm;
  if (read_ints(cacheFEPath(), fe) && read_ints(cacheFVVPath(), fvv) && read_ints(cacheFVMPath(), fvm) &&
      fvv.size() == fvm.size() && std::is_sorted(fvm.begin(), fvm.end())) {
    if (fe.size() >= E) edge_.assign(fe.begin(), fe.begin() + (long)E);
    vertex_ = std::move(fvv);
    vertexIds_ = std::move(fvm);
    return;
  }
  if (pathToRands.empty()) return;
  // distinct vertex ids, ascending; vertex i of that order takes value i
  // (src/core/gpu/data.cu:57-79)
  std::vector<int> ids(eloader->U());
  ids.insert(ids.end(), eloader->V().begin(), eloader->V().end());
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  std::vector<int> r;
  if (!read_ints_prefix(pathToRands, std::max(E, ids.size()), r)) return;
  if (r.size() >= E) edge_.assign(r.begin(), r.begin() + (long)E);
  if (r.size() >= ids.size()) {
    vertex_.assign(r.begin(), r.begin() + (long)ids.size());
    vertexIds_ = std::move(ids);
  }
  if (edge_.size() == E && !vertex_.empty() && std::filesystem::exists(cacheDir_)) {
    write_ints(cacheFEPath(), edge_);
    write_ints(cacheFVVPath(), vertex_);
    write_ints(cacheFVMPath(), vertexIds_);
  }
}

int FeatureLoader::vertexFeature(int id) const {
  auto it = std::lower_bound(vertexIds_.begin(), vertexIds_.end(), id);
  if (it == vertexIds_.end()) return 0;
  return vertex_[(size_t)(it - vertexIds_.begin())];
}

SubPartitionList divideList(const EdgeListLoader &eloader, int delta, int num) {
  if (num < 1) throw std::invalid_argument("divideList: num must be >= 1");
  const std::vector<int> &time = eloader.T();
  const size_t size = eloader.edgeListLength();
  SubPartitionList res(num * 2 - 1, SubPartition{0, 0, 0});
  const size_t chunk = size / num;
  for (int i = 0; i < num; i++) {
    res[i].beg = (int)(i * chunk);
    res[i].end = (int)((i + 1) * chunk);
  }
  res[num - 1].end = (int)size;
  res[num - 1].n = res[num - 1].end - res[num - 1].beg;
  for (int i = 0; i < num - 1; i++) {
    const int p = res[i].end;
    const int t = time[p];
    const long long lo = (long long)t - delta, hi = (long long)t + delta;
    const long loId = (long)(std::lower_bound(time.begin(), time.end(), lo) - time.begin()) - 1;
    const long hiId = (long)(std::lower_bound(time.begin(), time.end(), hi) - time.begin()) + 1;
    res[i + num].beg = (int)loId;
    res[i + num].end = (int)hiId;
    res[i + num].n = (int)(p - loId);
    res[i].n = (int)(loId - res[i].beg);
  }
  return res;
}

void removeMinor(HostGraphDataList &complete) { complete.resize((complete.size() + 1) / 2); }

void includeMinor(HostGraphDataList &major, HostGraphDataList &minor) {
  for (auto &m : minor) major.push_back(std::move(m));
  minor.clear();
}

GraphDataLoader::GraphDataLoader(const EdgeListLoader *eloader, const FeatureLoader *floader)
    : CacheDirectoryAccess(eloader->graphPath_, false), eloader_(eloader), floader_(floader),
      stem_(eloader->name_) {}

bool GraphDataLoader::isCached(size_t beg, size_t end) const {
  return std::filesystem::exists(cacheGraphDirPath(beg, end) / "Eg");
}

HostGraphData GraphDataLoader::loadGraphData(size_t beg, size_t end) const {
  HostGraphData res;
  const auto cpath = cacheGraphDirPath(beg, end);
  res.name = cpath.filename().string();
  res.beg = beg;
  res.end = end;
  bool ok = read_ints(cpath / "Eg", res.Eg) && read_ints(cpath / "inEdgesV", res.inEdgesV) &&
            read_ints(cpath / "outEdgesV", res.outEdgesV) && read_ints(cpath / "inEdgesR", res.inEdgesR) &&
            read_ints(cpath / "outEdgesR", res.outEdgesR) && read_ints(cpath / "Euid", res.Euid);
  if (!ok || res.Eg.size() % 3 || res.inEdgesR.empty())
    throw std::runtime_error("corrupt graph cache directory " + cpath.string());
  read_ints(cpath / "edgeFeatures", res.edgeFeatures);
  read_ints(cpath / "verticesFeatures", res.verticesFeatures);
  res.numEdges = res.Eg.size() / 3;
  res.numVertices = res.inEdgesR.size() - 1;
  res.totalBytes = calc_total_bytes(res.numEdges, res.numVertices);
  return res;
}

HostGraphData GraphDataLoader::createGraphData(size_t beg, size_t end, bool cache) const {
  if (end == 0) end = eloader_->edgeListLength();
  if (end > eloader_->edgeListLength() || beg > end)
    throw std::invalid_argument("createGraphData: bad edge range");
  if (cache && isCached(beg, end)) return loadGraphData(beg, end);
  HostGraphData res;
  res.name = cacheGraphDirPath(beg, end).filename().string();
  res.beg = beg;
  res.end = end;
  int64_t E = 0, V = 0;
  int *eg, *ov, *iv, *orr, *irr, *eu;
  check_evx(evx_graph_build_host(eloader_->U().data(), eloader_->V().data(), eloader_->T().data(),
                                 eloader_->IDS().data(), (int64_t)beg, (int64_t)end, &E, &V, &eg,
                                 &ov, &iv, &orr, &irr, &eu),
            "createGraphData");
  res.numEdges = (size_t)E;
  res.numVertices = (size_t)V;
  res.Eg = take_ints(eg, (size_t)(3 * E));
  res.outEdgesV = take_ints(ov, (size_t)E);
  res.inEdgesV = take_ints(iv, (size_t)E);
  res.outEdgesR = take_ints(orr, (size_t)(V + 1));
  res.inEdgesR = take_ints(irr, (size_t)(V + 1));
  res.Euid = take_ints(eu, (size_t)E);
  const auto &fe = floader_ ? floader_->edgeFeatures() : std::vector<int>();
  if (fe.size() >= end) res.edgeFeatures.assign(fe.begin() + (long)beg, fe.begin() + (long)end);
  if (floader_ && floader_->hasVertexFeatures()) {
    // relabeled vertex -> its input id -> feature (src/core/gpu/data.cu:200-216)
    res.verticesFeatures.assign((size_t)V, 0);
    const int *U = eloader_->U().data(), *Vv = eloader_->V().data();
    for (int64_t i = 0; i < E; i++) {
      res.verticesFeatures[(size_t)res.Eg[3 * i]] = floader_->vertexFeature(U[beg + i]);
      res.verticesFeatures[(size_t)res.Eg[3 * i + 1]] = floader_->vertexFeature(Vv[beg + i]);
    }
  }
  res.totalBytes = calc_total_bytes(res.numEdges, res.numVertices);
  if (cache) {
    const auto cpath = cacheGraphDirPath(beg, end);
    std::error_code ec;
    std::filesystem::create_directories(cpath, ec);
    if (!ec) {
      write_ints(cpath / "Eg", res.Eg);
      write_ints(cpath / "inEdgesV", res.inEdgesV);
      write_ints(cpath / "outEdgesV", res.outEdgesV);
      write_ints(cpath / "inEdgesR", res.inEdgesR);
      write_ints(cpath / "outEdgesR", res.outEdgesR);
      write_ints(cpath / "Euid", res.Euid);
      write_ints(cpath / "edgeFeatures", res.edgeFeatures);
      write_ints(cpath / "verticesFeatures", res.verticesFeatures);
    }
  }
  return res;
}

HostGraphDataList GraphDataLoader::createPartitionsData(const SubPartitionList &partitions) const {
  HostGraphDataList major = createPartitionsDataMajor(partitions);
  HostGraphDataList minor = createPartitionsDataMinor(partitions);
  includeMinor(major, minor);
  return major;
}

HostGraphDataList GraphDataLoader::createPartitionsDataMajor(const SubPartitionList &partitions) const {
  HostGraphDataList res;
  const size_t major = (partitions.size() + 1) / 2;
  for (size_t i = 0; i < major; i++) res.push_back(createGraphData(partitions[i].beg, partitions[i].end, true));
  return res;
}

HostGraphDataList GraphDataLoader::createPartitionsDataMinor(const SubPartitionList &partitions) const {
  HostGraphDataList res;
  const size_t major = (partitions.size() + 1) / 2;
  for (size_t i = major; i < partitions.size(); i++)
    res.push_back(createGraphData(partitions[i].beg, partitions[i].end, false));
  return res;
}

namespace {
struct GraphDataManagerImpl : GraphDataManager {
  int total_;
  explicit GraphDataManagerImpl(int total) : total_(total) {}
  std::vector<DeviceGraphData> allocBatch(int allDevices,
                                          const std::vector<const HostGraphData *> &hostGraphs) const override {
    std::vector<DeviceGraphData> res;
    for (int d = 0; d < allDevices; d++) {
      DeviceGraphData g;
      g.device = d;
      res.push_back(g);
    }
    (void)hostGraphs;
    return res;
  }
  DeviceGraphData alloc(int device, const HostGraphData *hostGraph) const override {
    DeviceGraphData g;
    g.device = device;
    if (hostGraph) {
      g.numEdges = hostGraph->numEdges;
      g.numVertices = hostGraph->numVertices;
    }
    return g;
  }
  void moveAsync(DeviceGraphData &s, const HostGraphData &h, int device) const override {
    evx_graph *gp = nullptr;
    check_evx(evx_graph_upload(device, (int64_t)h.numEdges, (int64_t)h.numVertices, h.Eg.data(),
                               h.outEdgesV.data(), h.inEdgesV.data(), h.outEdgesR.data(),
                               h.inEdgesR.data(), h.Euid.empty() ? nullptr : h.Euid.data(), nullptr,
                               &gp),
              "GraphDataManager::moveAsync");
    s.graph = std::shared_ptr<evx_graph>(gp, [](evx_graph *p) { evx_graph_free(p); });
    const bool vf = h.verticesFeatures.size() == h.numVertices && h.numVertices > 0;
    const bool ef = h.edgeFeatures.size() == h.numEdges && h.numEdges > 0;
    if (vf || ef)
      check_evx(evx_graph_set_features(gp, vf ? h.verticesFeatures.data() : nullptr,
                                       ef ? h.edgeFeatures.data() : nullptr),
                "GraphDataManager::moveAsync(features)");
    s.device = device;
    s.name = h.name;
    s.beg = h.beg;
    s.end = h.end;
    s.numEdges = h.numEdges;
    s.numVertices = h.numVertices;
    s.totalBytes = h.totalBytes;
  }
  void waitMove(int) const override {}  // evx_graph_upload completes before returning
};
}  // namespace

std::unique_ptr<GraphDataManager> MakeGraphDataManager(int totalDevice) {
  if (totalDevice < 1) throw std::invalid_argument("MakeGraphDataManager: need >= 1 device");
  return std::unique_ptr<GraphDataManager>(new GraphDataManagerImpl(totalDevice));
}

static void fill_motif(HostMotifData &m, int k, const int *mu, const int *mv, int nn) {
  m.numEdges = (size_t)k;
  m.numVertices = (size_t)nn;
  m.edges.clear();
  m.minfo.clear();
  for (int j = 0; j < k; j++) m.edges.push_back({mu[j], mv[j], j + 1});
  // src/core/cpu/data.cc:416-446
  int nodeMax = 1;
  for (int j = 1; j < k; j++) {
    MotifEdgeInfoV1 mi;
    const int u = mu[j], v = mv[j];
    if (u > nodeMax) {
      mi = {v, -u, nodeMax + 1, 0, true};
      nodeMax++;
    } else if (v > nodeMax) {
      mi = {u, -v, nodeMax + 1, 1, true};
      nodeMax++;
    } else {
      mi = {v, u, nodeMax + 1, -1, false};
    }
    m.minfo.push_back(mi);
  }
}

HostMotifData::HostMotifData(const std::filesystem::path &pathToMotif) {
  int k = 0, nn = 0, mu[EVX_MAX_MOTIF_EDGES], mv[EVX_MAX_MOTIF_EDGES];
  check_evx(evx_motif_parse(pathToMotif.string().c_str(), &k, mu, mv, &nn), "HostMotifData");
  name = pathToMotif.stem().string();
  fill_motif(*this, k, mu, mv, nn);
}

HostMotifData HostMotifData::fromText(const std::string &text, const std::string &nm) {
  int k = 0, nn = 0, mu[EVX_MAX_MOTIF_EDGES], mv[EVX_MAX_MOTIF_EDGES];
  check_evx(evx_motif_parse_text(text.c_str(), &k, mu, mv, &nn), "HostMotifData");
  HostMotifData m;
  m.name = nm;
  fill_motif(m, k, mu, mv, nn);
  return m;
}

DeviceJobData::DeviceJobData(const DeviceGraphData &deviceGraph, const HostMotifData &hostMotif) {
  if (!deviceGraph.graph) throw std::runtime_error("DeviceJobData: device graph not loaded");
  device = deviceGraph.device;
  graphNumEdges = deviceGraph.numEdges;
  graphNumVertices = deviceGraph.numVertices;
  motifNumEdges = hostMotif.numEdges;
  motifNumVertices = hostMotif.numVertices;
  graph = deviceGraph.graph;
  for (auto &e : hostMotif.edges) {
    mu.push_back(e.u);
    mv.push_back(e.v);
  }
  minfol_ = hostMotif.minfo;
}

MineJob::MineJob(const DeviceJobData *_data, int _delta, int _beg, int _end)
    : device(_data ? _data->device : -1), beg(_beg), end(_end), delta(_delta), data(_data) {
  if (!_data) throw std::invalid_argument("MineJob: null job data");
  // src/core/cpu/data.cc:452-457
  if (end == -1) end = (int)_data->graphNumEdges - (int)_data->motifNumEdges + 1;
}

}  // namespace data

// ------------------------------------------------------------- workers --

GPUWorker::GPUWorker(std::string type, int gpu, int sizeBlock)
    : type_(std::move(type)), gpu_(gpu), time_(0), sizeBlock_(sizeBlock), count_(0) {}
GPUWorker::~GPUWorker() {}

void GPUWorker::take(data::MineJob &job) { job_ = &job; }

int GPUWorker::numBlocks() { return job_ ? (job_->end + sizeBlock_ - 1) / sizeBlock_ : -1; }

unsigned long long GPUWorker::timed_run() {
  // src/core/cpu/data.cc:534-542: host microseconds around run()
  auto st = std::chrono::high_resolution_clock::now();
  auto res = run();
  auto ed = std::chrono::high_resolution_clock::now();
  time_ += (unsigned long long)std::chrono::duration_cast<std::chrono::microseconds>(ed - st).count();
  return res;
}

std::vector<int> GPUWorker::printEnum(int) { return {}; }
std::pair<int, int> GPUWorker::pause() { return {-1, -1}; }
void GPUWorker::configure(long long, unsigned) {}
void GPUWorker::setTuning(int, int, int, int, int) {}
double GPUWorker::lastDeviceMs() const { return 0.0; }
void GPUWorker::setConstraints(const evx_constraints *c) {
  if (c) throw std::runtime_error("this worker takes no query constraints");
}
int GPUWorker::lastKernelLaunches() const { return 0; }

GPUWorkerEVX::GPUWorkerEVX(int gpu, int sizeBlock) : GPUWorker("EVX", gpu, sizeBlock) {
  check_evx(evx_worker_create(gpu, nullptr, &w_), "getWorker");
}

GPUWorkerEVX::~GPUWorkerEVX() { evx_worker_destroy(w_); }

void GPUWorkerEVX::setConstraints(const evx_constraints *c) {
  hasCons_ = c != nullptr;
  if (c) cons_ = *c;
}

void GPUWorkerEVX::configure(long long enumCap, unsigned flags) {
  enumCap_ = enumCap;
  flags_ = flags;
}

void GPUWorkerEVX::setTuning(int block, int bps, int rpf, int steal, int minSplit) {
  check_evx(evx_worker_set_tuning(w_, block, bps, rpf, steal, minSplit), "setTuning");
  sizeBlock_ = block;
}

void GPUWorkerEVX::take(data::MineJob &job) {
  GPUWorker::take(job);
  const data::DeviceJobData *d = job.data;
  if (!d || !d->graph) throw std::runtime_error("take: job without device data");
  k_ = (int)d->mu.size();
  if (hasCons_)
    check_evx(evx_worker_take_constrained(w_, d->graph.get(), k_, d->mu.data(), d->mv.data(), job.delta,
                                          job.beg, job.end, enumCap_, flags_, &cons_),
              "take");
  else
    check_evx(evx_worker_take(w_, d->graph.get(), k_, d->mu.data(), d->mv.data(), job.delta, job.beg,
                              job.end, enumCap_, flags_),
              "take");
  bound_ = true;
}

unsigned long long GPUWorkerEVX::run() {
  if (!job_ || !bound_) throw std::runtime_error("run a GPU worker without a job");
  uint64_t c = 0;
  check_evx(evx_worker_run(w_, &c), "run");
  count_ = c;
  return count_;
}

void GPUWorkerEVX::update_job() {
  if (job_) job_->beg = job_->end;
}

std::vector<int> GPUWorkerEVX::printEnum(int n) {
  if (enumCap_ <= 0 || !bound_) return {};
  const long long f = std::min<long long>({(long long)n, (long long)count_, enumCap_});
  std::vector<int> vals((size_t)std::max<long long>(f, 0) * k_);
  int64_t wr = 0;
  if (f > 0) check_evx(evx_worker_enum_rows(w_, f, vals.data(), &wr), "printEnum");
  vals.resize((size_t)wr * k_);
  return vals;
}

double GPUWorkerEVX::lastDeviceMs() const {
  float ms = 0.f;
  int n = 0;
  evx_worker_last_stats(w_, &n, &ms);
  return ms;
}

int GPUWorkerEVX::lastKernelLaunches() const {
  float ms = 0.f;
  int n = 0;
  evx_worker_last_stats(w_, &n, &ms);
  return n;
}

LibHandle::LibHandle(const std::string &libpath) {
  handle = dlopen(libpath.c_str(), RTLD_LAZY);
  if (!handle) throw std::runtime_error(std::string("Load Lib Error: ") + dlerror());
  getWorker = (FactoryType)dlsym(handle, "getWorker");
  if (!getWorker) {
    std::string e = dlerror();
    dlclose(handle);
    handle = nullptr;
    throw std::runtime_error("query func Error: " + e);
  }
}

LibHandle::LibHandle(LibHandle &&rhs) noexcept : handle(rhs.handle), getWorker(rhs.getWorker) {
  rhs.handle = nullptr;
  rhs.getWorker = nullptr;
}

LibHandle &LibHandle::operator=(LibHandle &&rhs) noexcept {
  if (this != &rhs) {
    if (handle) dlclose(handle);
    handle = rhs.handle;
    getWorker = rhs.getWorker;
    rhs.handle = nullptr;
    rhs.getWorker = nullptr;
  }
  return *this;
}

LibHandle::~LibHandle() {
  if (handle) dlclose(handle);
}

std::string LibHandle::toString() const {
  std::ostringstream s;
  s << "handle: " << handle << ", factory: " << (void *)getWorker;
  return s.str();
}

static std::string lib_name_of(const std::string &libpath) {
  // lib<NAME>.so -> NAME (src/core/cpu/data.cc:611-625)
  std::string base = libpath.substr(libpath.find_last_of('/') == std::string::npos ? 0
                                                                                   : libpath.find_last_of('/') + 1);
  if (base.size() < 7 || base.compare(0, 3, "lib") != 0 || base.compare(base.size() - 3, 3, ".so") != 0)
    throw std::invalid_argument("plugin file must be named lib<NAME>.so: " + libpath);
  return base.substr(3, base.size() - 6);
}

void GPUWorkerLibManager::openLib(const std::string &libpath) {
  const std::string name = lib_name_of(libpath);
  table_.erase(name);
  table_.emplace(name, LibHandle(libpath));
}

void GPUWorkerLibManager::unloadLib(const std::string &lib) { table_.erase(lib); }

std::unique_ptr<GPUWorker> GPUWorkerLibManager::construct(const std::string &lib, int gpu) {
  auto it = table_.find(lib);
  if (it == table_.end()) throw std::out_of_range("library not opened: " + lib);
  GPUWorker *w = it->second.getWorker(gpu);
  if (!w) throw std::runtime_error("getWorker returned null: " + std::string(evx_last_error()));
  return std::unique_ptr<GPUWorker>(w);
}

std::string GPUWorkerLibManager::toString() const {
  std::ostringstream s;
  for (auto &e : table_) s << e.first << ": " << e.second.toString() << "\n";
  return s.str();
}

// ----------------------------------------------------------- executions --

SingleGPUExecution::SingleGPUExecution(const data::GraphDataManager *dataManager, int device)
    : device_(device), dataManager_(dataManager) {}

void SingleGPUExecution::formJobData() {
  if (hostGraph_ && hostMotif_) jobData_ = data::DeviceJobData(deviceGraph_, *hostMotif_);
}

void SingleGPUExecution::setHostGraph(const data::HostGraphData *hostGraph, int n) {
  if (!hostGraph) throw std::invalid_argument("setHostGraph: null graph");
  n_ = n;
  hostGraph_ = hostGraph;
  deviceGraph_ = dataManager_->alloc(device_, hostGraph_);
  dataManager_->moveAsync(deviceGraph_, *hostGraph_, device_);
  dataManager_->waitMove(device_);
  formJobData();
}

void SingleGPUExecution::setHostMotif(const data::HostMotifData *hostMotif) {
  hostMotif_ = hostMotif;
  formJobData();
}

void SingleGPUExecution::setWorker(GPUWorker *w) { w_ = w; }

unsigned long long SingleGPUExecution::run(int delta) {
  if (!w_) throw std::runtime_error("run: no worker set");
  if (!jobData_.graph) throw std::runtime_error("run: graph or motif not set");
  job_ = data::MineJob(&jobData_, delta, 0, n_);
  w_->take(job_);
  return w_->timed_run();
}

SingleGPUExecutionDiv::SingleGPUExecutionDiv(const data::GraphDataManager *dm, int device, int div)
    : SingleGPUExecution(dm, device), div_(div < 1 ? 1 : div) {}

unsigned long long SingleGPUExecutionDiv::run(int delta) {
  // src/core/cpu/data.cc:679-706: the root range split into div jobs
  if (!w_ || !jobData_.graph) throw std::runtime_error("run: graph, motif or worker not set");
  const int n = n_ < 0 ? (int)jobData_.graphNumEdges - (int)jobData_.motifNumEdges + 1 : n_;
  const int chunk = n / div_;
  unsigned long long res = 0;
  for (int i = 0; i < div_; i++) {
    job_ = data::MineJob(&jobData_, delta, i * chunk, i == div_ - 1 ? n : (i + 1) * chunk);
    w_->take(job_);
    res += w_->timed_run();
  }
  w_->count_ = res;
  return res;
}

void SingleGPURunBatch(const data::GraphDataManager *dataManager, data::HostGraphDataList &hostGraphs,
                       const data::HostMotifData *hostMotif, GPUWorker *w, int delta) {
  // src/core/cpu/data.cc:708-714: the partitions one after another
  unsigned long long total = 0;
  for (auto &g : hostGraphs) {
    SingleGPUExecution ex(dataManager, w->gpu_);
    ex.setHostGraph(&g);
    ex.setHostMotif(hostMotif);
    ex.setWorker(w);
    total += ex.run(delta);
  }
  w->count_ = total;
}

MultiGPUExecution::MultiGPUExecution(const data::GraphDataManager *dm, int deviceNum)
    : deviceNum_(deviceNum), dataManager_(dm) {
  if (deviceNum != 1)
    throw std::invalid_argument("multi-GPU execution is not on this path: one device only");
}

void MultiGPUExecution::setHostGraphs(const data::HostGraphDataList &hostGraphs,
                                      const data::SubPartitionList &ps) {
  hostGraphs_.clear();
  for (auto &g : hostGraphs) hostGraphs_.push_back(&g);
  parts_ = ps;
}

void MultiGPUExecution::setHostMotif(const data::HostMotifData *m) { hostMotif_ = m; }
void MultiGPUExecution::setWorkers(std::vector<GPUWorker *> &ws) { ws_ = ws; }

void MultiGPUExecution::run(int delta) {
  // One device: every partition's own root range (SubPartition::n) in turn.
  if (ws_.empty() || !hostMotif_) throw std::runtime_error("run: workers or motif not set");
  unsigned long long total = 0;
  for (size_t i = 0; i < hostGraphs_.size(); i++) {
    SingleGPUExecution ex(dataManager_, 0);
    const int n = i < parts_.size() ? parts_[i].n : -1;
    ex.setHostGraph(hostGraphs_[i], n);
    ex.setHostMotif(hostMotif_);
    ex.setWorker(ws_[0]);
    total += ex.run(delta);
  }
  ws_[0]->count_ = total;
}

unsigned long long allCount(std::vector<GPUWorker *> &ws) {
  unsigned long long r = 0;
  for (auto *w : ws) r += w->count();
  return r;
}

}  // namespace corelib
