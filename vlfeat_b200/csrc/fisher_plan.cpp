// Batched Fisher-encoding plans: the tensor-core encoder of
// vlb200_fisher_encode_batch_device bound to one batch layout, with an
// autotuner for its tile shapes and CUDA-graph capture of a whole encode.
// The reference has no counterpart; a plan computes what numImages calls of
// vl_fisher_encode (vl/fisher.c:548-579) compute.
#include <vector>

#include "engine.h"

extern "C" {
#include "vl/fisher.h"
#include "vlb200.h"
}

using vlb::i64;

struct _VlB200FisherPlan {
  vlb::TcFvPlan *plan = nullptr;
  vlb::DevModel<float> model;  // bound GMM (device pointers) with the plan's K and D
  bool hasModel = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long graphKernels = 0;  // kernel nodes of the captured graph

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    graphKernels = 0;
  }
  ~_VlB200FisherPlan() {
    drop_graph();
    vlb::tc_fv_plan_delete(plan);
  }
};

namespace {

template <typename F>
int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const vlb::Error &e) {
    vl_set_last_error(e.code, "%s", e.what());
    return e.code;
  } catch (const std::exception &e) {
    vl_set_last_error(VL_ERR_ALLOC, "%s", e.what());
    return VL_ERR_ALLOC;
  }
}

void need_model(const VlB200FisherPlan *p) {
  VLB_CHECK(p != nullptr, VL_ERR_BAD_ARG, "NULL plan");
  VLB_CHECK(p->hasModel, VL_ERR_BAD_ARG, "plan has no GMM: call vlb200_fisher_plan_set_gmm first");
}

vlb::TcFvConfig from_array(const vl_int64 c[5]) {
  vlb::TcFvConfig r;
  r.itemRows = c[0];
  r.statsMT = (int)c[1];
  r.statsStages = (int)c[2];
  r.estepStages = (int)c[3];
  r.rowBudget = c[4];
  return r;
}

}  // namespace

extern "C" {

VlB200FisherPlan *vlb200_fisher_plan_new(vl_size dimension, vl_size numClusters,
                                         vl_int64 const *offsets, vl_size numImages, int flags,
                                         int precision) {
  VlB200FisherPlan *out = nullptr;
  guarded([&] {
    VLB_CHECK(offsets != nullptr && offsets[0] >= 0, VL_ERR_BAD_ARG, "bad offsets");
    const int prec = vlb::resolve_precision(precision, false);
    auto *p = new VlB200FisherPlan();
    p->model.D = (i64)dimension;
    p->model.K = (i64)numClusters;
    try {
      p->plan = vlb::tc_fv_plan_new((i64)dimension, (i64)numClusters, (const i64 *)offsets,
                                    (i64)numImages, flags, prec, vlb::thread_stream());
    } catch (...) {
      delete p;
      throw;
    }
    out = p;
  });
  return out;
}

void vlb200_fisher_plan_delete(VlB200FisherPlan *plan) { delete plan; }

int vlb200_fisher_plan_set_gmm(VlB200FisherPlan *plan, float const *means, float const *covariances,
                               float const *priors) {
  return guarded([&] {
    VLB_CHECK(plan != nullptr && means && covariances && priors, VL_ERR_BAD_ARG, "NULL argument");
    plan->model.means = means;
    plan->model.covs = covariances;
    plan->model.priors = priors;
    plan->hasModel = true;
    plan->drop_graph();  // a captured graph holds the old pointers
  });
}

int vlb200_fisher_plan_execute(VlB200FisherPlan *plan, float *enc, float const *data,
                               vl_uint64 *numTerms, void *stream) {
  return guarded([&] {
    need_model(plan);
    vlb::tc_fv_plan_run(plan->plan, plan->model, data, enc, (unsigned long long *)numTerms,
                        vlb::pick_stream(stream));
  });
}

int vlb200_fisher_plan_execute_host(VlB200FisherPlan *plan, float *enc, float const *data,
                                    vl_uint64 *numTerms, void *stream) {
  return guarded([&] {
    need_model(plan);
    VLB_CHECK(enc != nullptr && data != nullptr, VL_ERR_BAD_ARG, "NULL argument");
    vlb::tc_fv_plan_run_host(plan->plan, plan->model, data, enc, (unsigned long long *)numTerms,
                             vlb::pick_stream(stream));
  });
}

int vlb200_fisher_plan_autotune(VlB200FisherPlan *plan, float *enc, float const *data,
                                vl_uint64 *numTerms, void *stream, double *bestMs) {
  return guarded([&] {
    need_model(plan);
    plan->drop_graph();  // the tables change with the configuration
    vlb::tc_fv_plan_autotune(plan->plan, plan->model, data, enc,
                             (unsigned long long *)numTerms, vlb::pick_stream(stream), bestMs);
  });
}

int vlb200_fisher_plan_get_config(VlB200FisherPlan const *plan, vl_int64 config[5]) {
  return guarded([&] {
    VLB_CHECK(plan != nullptr && config != nullptr, VL_ERR_BAD_ARG, "NULL argument");
    const vlb::TcFvConfig c = vlb::tc_fv_plan_config(plan->plan);
    config[0] = c.itemRows;
    config[1] = c.statsMT;
    config[2] = c.statsStages;
    config[3] = c.estepStages;
    config[4] = c.rowBudget;
  });
}

int vlb200_fisher_plan_set_config(VlB200FisherPlan *plan, vl_int64 const config[5], void *stream) {
  return guarded([&] {
    VLB_CHECK(plan != nullptr && config != nullptr, VL_ERR_BAD_ARG, "NULL argument");
    plan->drop_graph();
    vlb::tc_fv_plan_set_config(plan->plan, from_array(config), vlb::pick_stream(stream));
  });
}

int vlb200_fisher_plan_capture(VlB200FisherPlan *plan, float *enc, float const *data,
                               vl_uint64 *numTerms, void *stream) {
  return guarded([&] {
    need_model(plan);
    cudaStream_t s = vlb::pick_stream(stream);
    VLB_CHECK(s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread, VL_ERR_BAD_ARG,
              "graph capture needs a created stream (not the default stream)");
    const vlb::DevModel<float> &m = plan->model;
    plan->drop_graph();
    // One run outside the capture sizes every scratch buffer and sets the
    // kernels' shared-memory attributes, so the captured run allocates nothing.
    vlb::tc_fv_plan_run(plan->plan, m, data, enc, (unsigned long long *)numTerms, s);
    VLB_CUDA(cudaStreamSynchronize(s));
    const bool prof = vlb::profile_swap(false);  // no event timing inside the graph
    VLB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const unsigned long long l0 = vlb200_launch_count();
    try {
      vlb::tc_fv_plan_run(plan->plan, m, data, enc, (unsigned long long *)numTerms, s);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s, &g);
      if (g) cudaGraphDestroy(g);
      vlb::profile_swap(prof);
      throw;
    }
    const unsigned long long l1 = vlb200_launch_count();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    vlb::profile_swap(prof);
    VLB_CUDA(e);
    plan->graph = g;
    VLB_CUDA(cudaGraphInstantiate(&plan->exec, g, 0));
    plan->graphKernels = l1 - l0;
  });
}

int vlb200_fisher_plan_launch(VlB200FisherPlan *plan, void *stream) {
  return guarded([&] {
    VLB_CHECK(plan != nullptr && plan->exec != nullptr, VL_ERR_BAD_ARG,
              "plan has no captured graph: call vlb200_fisher_plan_capture first");
    VLB_CUDA(cudaGraphLaunch(plan->exec, vlb::pick_stream(stream)));
    vlb::count_launches(plan->graphKernels);
  });
}

int vlb200_fisher_plan_status(VlB200FisherPlan *plan, void *stream) {
  int r = 0;
  const int g = guarded([&] {
    VLB_CHECK(plan != nullptr, VL_ERR_BAD_ARG, "NULL plan");
    r = vlb::tc_fv_plan_error(plan->plan, vlb::pick_stream(stream));
  });
  return g ? g : r;
}

}  // extern "C"
