// reference_style.cu -- a functor written the way the reference's sample
// sources are (samples/hybrid_sssp/hybrid_sssp.cu:29-193 and :204-296): a
// template struct over <TValue, TBuffer, TWeight, UnusedData...> deriving
// from sepgraph::api::AppBase, members marked `override`, results returned
// as utils::pair, vertex ids as index_t, run by
// sepgraph::engine::Engine<TValue, TBuffer, TWeight, TAppImpl, Args...>
// through the driver calls the samples make.  It builds against
// include/sgs_app.cuh with SGS_APP_ACCEPT_OVERRIDE defined; the bodies are
// this project's own (shortest paths with strict (buffer, parent) updates).
#include <cstdint>
#include <string>
#include <utility>

#define SGS_APP_ACCEPT_OVERRIDE
#include "sgs_app.cuh"

#define IDENTITY_ELEMENT UINT32_MAX

namespace refstyle {

template <typename TValue, typename TBuffer, typename TWeight, typename... UnusedData>
struct SSSP : sepgraph::api::AppBase<TValue, TBuffer, TWeight> {
  index_t m_source_node;

  SSSP(index_t source_node) : m_source_node(source_node) {}

  __forceinline__ __device__ TValue GetInitValue(index_t node) const override {
    return static_cast<TValue>(IDENTITY_ELEMENT);
  }

  __forceinline__ __device__ TBuffer GetInitBuffer(index_t node) const override {
    return node == m_source_node ? 0 : IDENTITY_ELEMENT;
  }

  __forceinline__ __host__ __device__ TBuffer GetIdentityElement() const override { return IDENTITY_ELEMENT; }

  __forceinline__ __device__ utils::pair<TBuffer, bool> CombineValueBuffer(index_t node, TValue *p_value,
                                                                           TBuffer *p_buffer) override {
    TBuffer buffer = *p_buffer;
    bool schedule = *p_value > buffer;
    if (schedule) *p_value = buffer;
    return utils::pair<TBuffer, bool>(buffer, schedule);
  }

  __forceinline__ __device__ int AccumulateBuffer(index_t src, index_t dst, TWeight weight, TValue *p_parent,
                                                  TBuffer *p_buffer, TBuffer buffer) override {
    if (buffer == IDENTITY_ELEMENT) return this->ACCUMULATE_FAILURE_CONTINUE;
    const uint64_t next = (uint64_t)buffer + weight;
    if (next >= IDENTITY_ELEMENT) return this->ACCUMULATE_FAILURE_CONTINUE;
    return sgs::api::min_with_parent(p_parent, p_buffer, (TBuffer)next, src)
               ? this->ACCUMULATE_SUCCESS_CONTINUE
               : this->ACCUMULATE_FAILURE_CONTINUE;
  }

  __forceinline__ __device__ int AccumulateBuffer_del(index_t src, index_t dst, TValue *p_parent,
                                                      TBuffer *p_buffer, TValue *p_value) override {
    if (*(volatile TValue *)p_parent == src) {
      *reinterpret_cast<unsigned long long *>(p_parent) = ~0ull;  // buffer and parent reset together
      *p_value = IDENTITY_ELEMENT;
      this->m_vcsr_graph.vertices_[dst].deletion = true;
    }
    return 1;
  }

  __forceinline__ __device__ bool IsActiveNode(index_t node, TBuffer buffer, TValue value) const override {
    return buffer < value;
  }
};

}  // namespace refstyle

extern "C" {

// The samples' driver sequence on files in the reference's formats: load the
// graph, InitGraph(source), Start, get_update_file, then per snapshot
// del_edge + add_edge; values after the last snapshot into out (nv u32).
__attribute__((visibility("default"))) int sgs_sample_refstyle_sssp(const char *graphfile, const char *sizes,
                                                                    const char *updates, uint32_t source,
                                                                    uint32_t snapshots, uint32_t *out,
                                                                    uint32_t cap) {
  try {
    sgs_config cfg;
    sgs_config_default(&cfg);
    cfg.weight_mode = SGS_W_SYNTH;  // the reference's per-edge (u+v)%128+1
    typedef sepgraph::engine::Engine<uint32_t, uint32_t, uint32_t, refstyle::SSSP, index_t> HybridEngine;
    HybridEngine engine(&cfg);
    engine.LoadGraph(std::string(graphfile));
    engine.InitGraph(source);
    engine.Start();
    engine.compute_hot_vertices_sssp();
    engine.confirm_candidate_batch();
    engine.LoadCache();
    engine.get_update_file(sizes, updates);
    std::pair<index_t, index_t> local_begin(0, 0);
    for (index_t k = 0; k < snapshots; ++k) {
      engine.del_edge(local_begin, k);
      engine.add_edge(local_begin, k);
      engine.LoadCache();
    }
    engine.GatherValue();
    const auto &values = engine.GetGraphDatum().host_value;
    if (values.size() > cap) throw sgs::Error(SGS_ERR_INVALID, "output buffer too small");
    for (size_t i = 0; i < values.size(); ++i) out[i] = values[i];
    return SGS_OK;
  } catch (const sgs::Error &e) {
    sgs_set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    sgs_set_last_error(e.what());
    return SGS_ERR_CUDA;
  }
}

}  // extern "C"
