// LinearHSC : IterativeSolver -- the libuipc linear-system plugin, with its body
// replaced by calls into libhsc_b200.so through the C ABI (include/hsc_c_api.h).
//
// It keeps the reference plugin's contract (reproduction/hsc_backend/linear_hsc.cu):
//   * do_build (linear_hsc.cu:172-193): opt out with SimSystemException unless
//     linear_system/solver == "linear_hsc"; read the same linear_system/hsc/*
//     keys and linear_system/tol_rate;
//   * do_solve (linear_hsc.cu:344-436): solve on the SolvingInfo views, report
//     the iteration count, append the hsc_stats.jsonl record (:420-431) and
//     raise UIPC_ASSERT on the statuses the reference asserts on (no fallback).
// Built against libuipc's headers in libuipc, and against the minimal mock in
// uipc_mock/ here.
#include <cstdio>
#include <fstream>
#include <string>

#include <affine_body/abd_linear_subsystem.h>
#include <finite_element/fem_linear_subsystem.h>
#include <linear_system/iterative_solver.h>
#include <sim_engine.h>

#include "hsc_c_api.h"

namespace uipc::backend::cuda {

class LinearHSC final : public IterativeSolver {
  public:
    using IterativeSolver::IterativeSolver;
    ~LinearHSC() override {
        if (ctx) hsc_destroy(ctx);
    }
    const hsc_stats& last_stats() const { return stats; }

  private:
    ABDLinearSubsystem* abd = nullptr;
    FEMLinearSubsystem* fem = nullptr;
    GlobalTrajectoryFilter* contacts = nullptr;  // active contact counts for the record (linear_hsc.cu:179)
    hsc_ctx* ctx = nullptr;
    hsc_options opt{};
    hsc_stats stats{};

    template <class T> T key(const char* name, T fallback) {
        auto a = world().scene().config().find<T>(name);
        return a ? a->view()[0] : fallback;
    }

    void do_build(BuildInfo&) override {
        auto attr = world().scene().config().find<std::string>("linear_system/solver");
        if (!attr || attr->view()[0] != "linear_hsc") throw SimSystemException("LinearHSC unused");
        abd = &require<ABDLinearSubsystem>();
        fem = &require<FEMLinearSubsystem>();
        contacts = &require<GlobalTrajectoryFilter>();
        hsc_options_reference(&opt);  // linear_hsc.cu:162-164, integration.patch:33-54
        opt.max_rank = key<IndexT>("linear_system/hsc/max_rank", opt.max_rank);
        opt.neumann_order = key<IndexT>("linear_system/hsc/neumann_order", opt.neumann_order);
        opt.max_iter = key<IndexT>("linear_system/hsc/max_iter", opt.max_iter);
        opt.omega = key<Float>("linear_system/hsc/omega", opt.omega);
        opt.abd_inverse = key<IndexT>("linear_system/hsc/adaptive_abd_inverse", 1) ? HSC_ABD_ADAPTIVE : HSC_ABD_NEUMANN;
        opt.abd_inverse_tol = key<Float>("linear_system/hsc/abd_inverse_tol", opt.abd_inverse_tol);
        opt.full_residual_limit = key<Float>("linear_system/hsc/full_residual_limit", opt.full_residual_limit);
        opt.tol = key<Float>("linear_system/tol_rate", opt.tol);
        UIPC_ASSERT(opt.max_rank > 0 && opt.neumann_order > 0 && opt.max_iter > 0 && opt.omega > 0 &&
                        opt.omega <= 1,
                    "Invalid HSC parameters");
        const int rc = hsc_create(&opt, &ctx);
        UIPC_ASSERT(rc == HSC_OK, "LinearHSC: hsc_create failed (" + std::to_string(rc) + ")");
    }

    void do_solve(GlobalLinearSystem::SolvingInfo& info) override {
        auto A = info.A();
        hsc_bcoo3 M{A.row_indices().data(), A.col_indices().data(),
                    reinterpret_cast<const double*>(A.values().data()), (int64_t)A.triplet_count(),
                    (int32_t)A.total_rows()};
        hsc_dof_layout L{(int32_t)abd->dof_offset(), (int32_t)abd->dof_count(), (int32_t)fem->dof_offset(),
                         (int32_t)fem->dof_count()};
        const int rc = hsc_solve(ctx, &M, &L, info.b().buffer_view().data(), info.x().buffer_view().data(),
                                 nullptr, &stats);
        info.iter_count(stats.pcg_iterations);
        append_record(rc);
        UIPC_ASSERT(rc == HSC_OK, std::string("HSC: ") + hsc_last_error(ctx) + ". No fallback.");
    }

    void append_record(int rc) {
        // active contacts as the reference counts them (linear_hsc.cu:410-414): simplex pairs
        // PT + EE + PE + PP, vertex-half-plane pairs PH
        size_t mesh_contacts = 0, ground_contacts = 0;
        if (auto sf = contacts->find<SimplexTrajectoryFilter>())
            mesh_contacts = sf->PTs().size() + sf->EEs().size() + sf->PEs().size() + sf->PPs().size();
        if (auto gf = contacts->find<VertexHalfPlaneTrajectoryFilter>()) ground_contacts = gf->PHs().size();
        std::ofstream out(workspace() + "/hsc_stats.jsonl", std::ios::app);
        char buf[2048];
        std::snprintf(buf, sizeof buf,
                      "{\"frame\":%zu,\"newton\":%zu,\"fem_dofs\":%d,\"abd_dofs\":%d,\"active_fem_dofs\":%d,"
                      "\"rank\":%d,\"aca_relative_error\":%.17g,\"pcg_iterations\":%d,"
                      "\"schur_relative_residual\":%.17g,\"full_relative_residual\":%.17g,\"setup_ms\":%.6g,"
                      "\"total_ms\":%.6g,\"active_mesh_contacts\":%zu,\"active_ground_contacts\":%zu,"
                      "\"adaptive_abd_inverse\":%s,\"neumann_doublings\":%d,\"abd_inverse_residual\":%.17g,"
                      "\"full_residual_limit\":%.17g,\"accepted\":%s,\"solver\":\"linear_hsc\",\"fallback\":%s,"
                      "\"precision_mode\":\"%s\",\"preconditioner\":\"%s\",\"refinement_steps\":%d,"
                      "\"pcg_ms\":%.6g,\"lanczos_min\":%.17g,\"lanczos_max\":%.17g}\n",
                      engine().frame, engine().newton, stats.fem_dofs, stats.abd_dofs, stats.active_fem_dofs,
                      stats.rank, stats.aca_relative_error, stats.pcg_iterations, stats.schur_relative_residual,
                      stats.full_relative_residual, stats.setup_ms, stats.total_ms, mesh_contacts, ground_contacts,
                      opt.abd_inverse == HSC_ABD_ADAPTIVE ? "true" : "false", stats.neumann_doublings,
                      stats.abd_inverse_residual, opt.full_residual_limit, rc == HSC_OK ? "true" : "false",
                      stats.fallback ? "true" : "false",
                      stats.precision == HSC_BF16 ? "bf16" : stats.precision == HSC_FP32 ? "fp32" : "fp64",
                      stats.preconditioner == HSC_PRECOND_POLY ? "polynomial" : "neumann", stats.refinement_steps,
                      stats.pcg_ms, stats.lanczos_min, stats.lanczos_max);
        out << buf;
    }
};
REGISTER_SIM_SYSTEM(LinearHSC);

}  // namespace uipc::backend::cuda
