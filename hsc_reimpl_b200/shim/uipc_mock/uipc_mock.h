// Minimal stand-in for the libuipc types the LinearHSC plugin touches, so the
// shim compiles and runs here without libuipc (not vendored).  Names and
// signatures follow the libuipc call sites used by the reference plugin
// (reproduction/hsc_backend/linear_hsc.cu:153-437,
//  upstream/src/backends/cuda/linear_system/iterative_solver.h:8-53,
//  global_linear_system.h:347-365).  Only what the plugin uses is modelled.
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace uipc {
using IndexT = int32_t;
using SizeT = std::size_t;
using Float = double;

struct AssertionError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
#define UIPC_ASSERT(cond, msg)                                         \
    do {                                                               \
        if (!(cond)) throw ::uipc::AssertionError(std::string(msg));   \
    } while (0)

namespace backend::cuda {

struct SimSystemException : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// scene config: find<T>(key)->view()[0]
class Config {
  public:
    template <class T> struct Attr {
        std::vector<T> v;
        const std::vector<T>& view() const { return v; }
    };
    template <class T> std::shared_ptr<Attr<T>> find(const std::string& key) const;
    std::map<std::string, std::string> strs;
    std::map<std::string, double> nums;
};
template <> inline std::shared_ptr<Config::Attr<std::string>> Config::find<std::string>(const std::string& key) const {
    auto it = strs.find(key);
    if (it == strs.end()) return nullptr;
    return std::make_shared<Attr<std::string>>(Attr<std::string>{{it->second}});
}
template <> inline std::shared_ptr<Config::Attr<IndexT>> Config::find<IndexT>(const std::string& key) const {
    auto it = nums.find(key);
    if (it == nums.end()) return nullptr;
    return std::make_shared<Attr<IndexT>>(Attr<IndexT>{{(IndexT)it->second}});
}
template <> inline std::shared_ptr<Config::Attr<Float>> Config::find<Float>(const std::string& key) const {
    auto it = nums.find(key);
    if (it == nums.end()) return nullptr;
    return std::make_shared<Attr<Float>>(Attr<Float>{{it->second}});
}
struct Scene {
    Config cfg;
    Config& config() { return cfg; }
};
struct World {
    Scene sc;
    Scene& scene() { return sc; }
};

namespace cuda_tool {
template <class T> struct BufferView {
    T* p;
    SizeT n;
    T* data() const { return p; }
    SizeT size() const { return n; }
};
template <class T> struct DenseVectorView {
    T* p;
    SizeT n;
    SizeT size() const { return n; }
    BufferView<T> buffer_view() const { return {p, n}; }
};
template <class T> struct CDenseVectorView {
    const T* p;
    SizeT n;
    SizeT size() const { return n; }
    BufferView<const T> buffer_view() const { return {p, n}; }
};
template <class T, int N> struct CBCOOMatrixView {
    const int* rows;
    const int* cols;
    const T* vals;  // N*N per triplet, column-major (Eigen::Matrix<T,N,N>)
    SizeT count;
    SizeT nrows;
    BufferView<const int> row_indices() const { return {rows, count}; }
    BufferView<const int> col_indices() const { return {cols, count}; }
    BufferView<const T> values() const { return {vals, count * N * N}; }
    SizeT triplet_count() const { return count; }
    SizeT total_rows() const { return nrows; }
};
}  // namespace cuda_tool

struct ABDLinearSubsystem {
    IndexT off = 0, cnt = 0;
    IndexT dof_offset() const { return off; }
    IndexT dof_count() const { return cnt; }
};
struct FEMLinearSubsystem {
    IndexT off = 0, cnt = 0;
    IndexT dof_offset() const { return off; }
    IndexT dof_count() const { return cnt; }
};

struct GlobalLinearSystem {
    class SolvingInfo {
      public:
        cuda_tool::DenseVectorView<Float> m_x;
        cuda_tool::CDenseVectorView<Float> m_b;
        cuda_tool::CBCOOMatrixView<Float, 3> m_A;
        SizeT m_iters = 0;
        cuda_tool::DenseVectorView<Float> x() { return m_x; }
        cuda_tool::CDenseVectorView<Float> b() { return m_b; }
        cuda_tool::CBCOOMatrixView<Float, 3> A() const { return m_A; }
        void iter_count(SizeT n) { m_iters = n; }
    };
};

// the contact filters the plugin counts for its record (sizes only): simplex pairs PT, EE, PE, PP
// and vertex-half-plane pairs PH; GlobalTrajectoryFilter::find<T>() is null for a filter the scene
// does not have
struct Count {
    SizeT n = 0;
    SizeT size() const { return n; }
};
struct SimplexTrajectoryFilter {
    SizeT pt = 0, ee = 0, pe = 0, pp = 0;
    Count PTs() const { return {pt}; }
    Count EEs() const { return {ee}; }
    Count PEs() const { return {pe}; }
    Count PPs() const { return {pp}; }
};
struct VertexHalfPlaneTrajectoryFilter {
    SizeT ph = 0;
    Count PHs() const { return {ph}; }
};
struct GlobalTrajectoryFilter {
    SimplexTrajectoryFilter* simplex = nullptr;
    VertexHalfPlaneTrajectoryFilter* half_plane = nullptr;
    template <class T> T* find();
};
template <> inline SimplexTrajectoryFilter* GlobalTrajectoryFilter::find<SimplexTrajectoryFilter>() { return simplex; }
template <> inline VertexHalfPlaneTrajectoryFilter* GlobalTrajectoryFilter::find<VertexHalfPlaneTrajectoryFilter>() {
    return half_plane;
}

// the engine side the plugin reaches through SimSystem
struct Engine {
    World w;
    ABDLinearSubsystem abd;
    FEMLinearSubsystem fem;
    GlobalTrajectoryFilter contacts;
    std::string workspace = ".";
    SizeT frame = 0, newton = 0;
};

class SimSystem {
  public:
    explicit SimSystem(Engine& e) : m_engine(e) {}
    virtual ~SimSystem() = default;

  protected:
    World& world() { return m_engine.w; }
    template <class T> T& require();
    std::string workspace() const { return m_engine.workspace; }
    Engine& engine() { return m_engine; }
    Engine& m_engine;
};
template <> inline ABDLinearSubsystem& SimSystem::require<ABDLinearSubsystem>() { return m_engine.abd; }
template <> inline FEMLinearSubsystem& SimSystem::require<FEMLinearSubsystem>() { return m_engine.fem; }
template <> inline GlobalTrajectoryFilter& SimSystem::require<GlobalTrajectoryFilter>() { return m_engine.contacts; }

class IterativeSolver : public SimSystem {
  public:
    using SimSystem::SimSystem;
    class BuildInfo {};
    void build() {
        BuildInfo bi;
        do_build(bi);
    }
    void solve(GlobalLinearSystem::SolvingInfo& info) { do_solve(info); }

  protected:
    virtual void do_build(BuildInfo& info) = 0;
    virtual void do_solve(GlobalLinearSystem::SolvingInfo& info) = 0;
};

#define REGISTER_SIM_SYSTEM(T) \
    inline std::unique_ptr<::uipc::backend::cuda::IterativeSolver> make_##T(::uipc::backend::cuda::Engine& e) { return std::make_unique<T>(e); }

}  // namespace backend::cuda
}  // namespace uipc
