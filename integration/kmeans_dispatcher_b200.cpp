// oneDAL host-policy dispatchers for k-means Lloyd (dense) backed by the B200
// library (include/onedal_b200_kmeans.h). Compiled against the unchanged
// oneDAL headers in place of the reference's host-policy instantiations of
// cpp/oneapi/dal/algo/kmeans/detail/train_ops.cpp:35-42 and
// detail/infer_ops.cpp:37-43; everything above them (descriptor, tables,
// pre/post-condition checks of detail/train_ops.hpp:40-84) stays oneDAL's.
#include "oneapi/dal/algo/kmeans/detail/infer_ops.hpp"
#include "oneapi/dal/algo/kmeans/detail/train_ops.hpp"
#include "oneapi/dal/detail/common.hpp"
#include "oneapi/dal/detail/error_messages.hpp"
#include "oneapi/dal/detail/policy.hpp"
#include "oneapi/dal/detail/spmd_policy.hpp"
#include "oneapi/dal/exceptions.hpp"
#include "oneapi/dal/table/csr_accessor.hpp"
#include "oneapi/dal/table/homogen.hpp"
#include "oneapi/dal/table/row_accessor.hpp"

#include "onedal_b200_kmeans.h"

#include <type_traits>

namespace oneapi::dal::kmeans::detail::v1 {

namespace {

// One context (CUDA stream + workspace) per host thread; the C ABI context is
// not thread-safe.
kmb_context *thread_context() {
    thread_local struct Holder {
        kmb_context *ctx = nullptr;
        ~Holder() {
            if (ctx) kmb_context_destroy(ctx);
        }
    } holder;
    if (!holder.ctx) {
        const int rc = kmb_context_create(0, &holder.ctx);
        if (rc != KMB_OK) {
            holder.ctx = nullptr;
            throw internal_error(kmb_status_string(rc));
        }
    }
    return holder.ctx;
}

// kmb_status -> the exception types oneDAL raises for the same failures
// (cpp/oneapi/dal/backend/interop/error_converter.cpp:136-254).
void check(kmb_context *ctx, int status) {
    switch (status) {
        case KMB_OK: return;
        case KMB_EINVAL: throw invalid_argument(kmb_context_last_error(ctx));
        case KMB_ENOMEM: throw host_bad_alloc();
        case KMB_ETOO_MANY_EMPTY: throw domain_error(kmb_status_string(status));
        default: throw internal_error(kmb_context_last_error(ctx));
    }
}

template <typename F>
constexpr int dtype_of = std::is_same_v<F, float> ? KMB_F32 : KMB_F64;

}  // namespace

template <typename F>
struct train_ops_dispatcher<dal::detail::host_policy, F, method::lloyd_dense, task::clustering> {
    train_result<task::clustering> operator()(const dal::detail::host_policy &,
                                              const descriptor_base<task::clustering> &desc,
                                              const train_input<task::clustering> &input) const {
        const table &data = input.get_data();
        const std::int64_t n = data.get_row_count();
        const std::int64_t d = data.get_column_count();
        const std::int64_t k = desc.get_cluster_count();
        const auto x = row_accessor<const F>(data).pull({ 0, -1 });
        kmb_context *ctx = thread_context();
        array<F> c0;
        if (input.get_initial_centroids().has_data()) {
            c0 = row_accessor<const F>(input.get_initial_centroids()).pull({ 0, -1 });
        }
        else {
            // oneDAL's default when no initial centroids are given: k-means++ with one
            // trial and seed 777777 (detail/train_init_centroids.hpp:47-74)
            c0 = array<F>::empty(k * d);
            check(ctx, kmb_init_plusplus(ctx, dtype_of<F>, KMB_MEM_HOST, x.get_data(), n, d, k,
                                         KMB_PLUSPLUS_DEFAULT_SEED, c0.get_mutable_data()));
        }
        auto centroids = array<F>::empty(k * d);
        auto responses = array<std::int32_t>::empty(n);
        kmb_params p{ k, desc.get_max_iteration_count(), desc.get_accuracy_threshold(), KMB_FORM_AUTO, 0 };
        double objective = 0.0;
        std::int64_t iterations = 0;
        check(ctx, kmb_train(ctx, dtype_of<F>, KMB_MEM_HOST, x.get_data(), n, d, c0.get_data(), &p,
                             centroids.get_mutable_data(), responses.get_mutable_data(), &objective, &iterations,
                             nullptr));
        return train_result<task::clustering>{}
            .set_model(model<task::clustering>{}.set_centroids(
                dal::detail::homogen_table_builder{}.reset(centroids, k, d).build()))
            .set_responses(dal::detail::homogen_table_builder{}.reset(responses, n, 1).build())
            .set_iteration_count(iterations)
            .set_objective_function_value(objective);
    }
};

template <typename F>
struct infer_ops_dispatcher<dal::detail::host_policy, F, method::lloyd_dense, task::clustering> {
    infer_result<task::clustering> operator()(const dal::detail::host_policy &,
                                              const descriptor_base<task::clustering> &desc,
                                              const infer_input<task::clustering> &input) const {
        const table &data = input.get_data();
        const table &c = input.get_model().get_centroids();
        const std::int64_t n = data.get_row_count();
        const std::int64_t d = data.get_column_count();
        const std::int64_t k = c.get_row_count();
        const auto x = row_accessor<const F>(data).pull({ 0, -1 });
        const auto cc = row_accessor<const F>(c).pull({ 0, -1 });
        const bool want_obj =
            desc.get_result_options().test(result_options::compute_exact_objective_function);
        auto responses = array<std::int32_t>::empty(n);
        double objective = 0.0;
        kmb_context *ctx = thread_context();
        check(ctx, kmb_infer(ctx, dtype_of<F>, KMB_MEM_HOST, x.get_data(), n, d, cc.get_data(), k, KMB_FORM_AUTO,
                             want_obj ? 1 : 0, responses.get_mutable_data(), &objective, nullptr));
        auto result = infer_result<task::clustering>{}.set_result_options(desc.get_result_options());
        result.set_responses(dal::detail::homogen_table_builder{}.reset(responses, n, 1).build());
        if (want_obj) result.set_objective_function_value(objective);
        return result;
    }
};

// method::lloyd_csr: the data table is a csr_table, pulled zero-based; centroids
// stay dense (detail/train_ops.cpp:41-42, detail/infer_ops.cpp:42-43).
template <typename F>
struct train_ops_dispatcher<dal::detail::host_policy, F, method::lloyd_csr, task::clustering> {
    train_result<task::clustering> operator()(const dal::detail::host_policy &,
                                              const descriptor_base<task::clustering> &desc,
                                              const train_input<task::clustering> &input) const {
        const table &data = input.get_data();
        const std::int64_t n = data.get_row_count();
        const std::int64_t d = data.get_column_count();
        const std::int64_t k = desc.get_cluster_count();
        if (data.get_kind() != csr_table::kind()) throw invalid_argument("method::lloyd_csr takes a csr_table");
        const auto [vals, cols, offs] =
            csr_accessor<const F>(static_cast<const csr_table &>(data)).pull({ 0, -1 }, sparse_indexing::zero_based);
        kmb_context *ctx = thread_context();
        array<F> c0;
        if (input.get_initial_centroids().has_data()) {
            c0 = row_accessor<const F>(input.get_initial_centroids()).pull({ 0, -1 });
        }
        else {
            // the default for lloyd_csr: plusPlusCSR, one trial, seed 777777
            // (detail/train_init_centroids.hpp:39-74)
            c0 = array<F>::empty(k * d);
            check(ctx, kmb_init_plusplus_csr(ctx, dtype_of<F>, KMB_MEM_HOST, vals.get_data(), cols.get_data(),
                                             offs.get_data(), n, d, 0, k, KMB_PLUSPLUS_DEFAULT_SEED,
                                             c0.get_mutable_data()));
        }
        auto centroids = array<F>::empty(k * d);
        auto responses = array<std::int32_t>::empty(n);
        kmb_params p{ k, desc.get_max_iteration_count(), desc.get_accuracy_threshold(), KMB_FORM_PLAIN, 0 };
        double objective = 0.0;
        std::int64_t iterations = 0;
        check(ctx, kmb_train_csr(ctx, dtype_of<F>, KMB_MEM_HOST, vals.get_data(), cols.get_data(), offs.get_data(),
                                 n, d, 0, c0.get_data(), &p, centroids.get_mutable_data(),
                                 responses.get_mutable_data(), &objective, &iterations, nullptr));
        return train_result<task::clustering>{}
            .set_model(model<task::clustering>{}.set_centroids(
                dal::detail::homogen_table_builder{}.reset(centroids, k, d).build()))
            .set_responses(dal::detail::homogen_table_builder{}.reset(responses, n, 1).build())
            .set_iteration_count(iterations)
            .set_objective_function_value(objective);
    }
};

template <typename F>
struct infer_ops_dispatcher<dal::detail::host_policy, F, method::lloyd_csr, task::clustering> {
    infer_result<task::clustering> operator()(const dal::detail::host_policy &,
                                              const descriptor_base<task::clustering> &desc,
                                              const infer_input<task::clustering> &input) const {
        const table &data = input.get_data();
        const table &c = input.get_model().get_centroids();
        const std::int64_t n = data.get_row_count();
        const std::int64_t d = data.get_column_count();
        const std::int64_t k = c.get_row_count();
        if (data.get_kind() != csr_table::kind()) throw invalid_argument("method::lloyd_csr takes a csr_table");
        const auto [vals, cols, offs] =
            csr_accessor<const F>(static_cast<const csr_table &>(data)).pull({ 0, -1 }, sparse_indexing::zero_based);
        const auto cc = row_accessor<const F>(c).pull({ 0, -1 });
        const bool want_obj =
            desc.get_result_options().test(result_options::compute_exact_objective_function);
        auto responses = array<std::int32_t>::empty(n);
        double objective = 0.0;
        kmb_context *ctx = thread_context();
        check(ctx, kmb_infer_csr(ctx, dtype_of<F>, KMB_MEM_HOST, vals.get_data(), cols.get_data(), offs.get_data(), n,
                                 d, 0, cc.get_data(), k, want_obj ? 1 : 0, responses.get_mutable_data(), &objective));
        auto result = infer_result<task::clustering>{}.set_result_options(desc.get_result_options());
        result.set_responses(dal::detail::homogen_table_builder{}.reset(responses, n, 1).build());
        if (want_obj) result.set_objective_function_value(objective);
        return result;
    }
};

template struct ONEDAL_EXPORT
    train_ops_dispatcher<dal::detail::host_policy, float, method::lloyd_csr, task::clustering>;
template struct ONEDAL_EXPORT
    train_ops_dispatcher<dal::detail::host_policy, double, method::lloyd_csr, task::clustering>;
template struct ONEDAL_EXPORT
    infer_ops_dispatcher<dal::detail::host_policy, float, method::lloyd_csr, task::clustering>;
template struct ONEDAL_EXPORT
    infer_ops_dispatcher<dal::detail::host_policy, double, method::lloyd_csr, task::clustering>;

// SPMD train (dal::preview::train(comm, ...), cpp/oneapi/dal/train.hpp:43-50) on
// the host: the reference instantiates these next to the host-policy ones
// (detail/train_ops.cpp:35-37) and its single-node CPU kernel dispatcher answers
// them with unimplemented(spmd_version_of_algorithm_is_not_implemented)
// (cpp/oneapi/dal/backend/dispatcher.hpp:186-199). The same answer here keeps
// every symbol and behaviour a client links against; row-sharded multi-GPU
// training runs through kmb_partial_sums / kmb_finalize_centroids instead.
template <typename F, typename M>
struct train_ops_dispatcher<dal::detail::spmd_host_policy, F, M, task::clustering> {
    train_result<task::clustering> operator()(const dal::detail::spmd_host_policy &,
                                              const descriptor_base<task::clustering> &,
                                              const train_input<task::clustering> &) const {
        throw unimplemented{ dal::detail::error_messages::spmd_version_of_algorithm_is_not_implemented() };
    }
};

template struct ONEDAL_EXPORT
    train_ops_dispatcher<dal::detail::spmd_host_policy, float, method::lloyd_dense, task::clustering>;
template struct ONEDAL_EXPORT
    train_ops_dispatcher<dal::detail::spmd_host_policy, double, method::lloyd_dense, task::clustering>;
template struct ONEDAL_EXPORT
    train_ops_dispatcher<dal::detail::spmd_host_policy, float, method::lloyd_csr, task::clustering>;
template struct ONEDAL_EXPORT
    train_ops_dispatcher<dal::detail::spmd_host_policy, double, method::lloyd_csr, task::clustering>;

template struct ONEDAL_EXPORT
    train_ops_dispatcher<dal::detail::host_policy, float, method::lloyd_dense, task::clustering>;
template struct ONEDAL_EXPORT
    train_ops_dispatcher<dal::detail::host_policy, double, method::lloyd_dense, task::clustering>;
template struct ONEDAL_EXPORT
    infer_ops_dispatcher<dal::detail::host_policy, float, method::lloyd_dense, task::clustering>;
template struct ONEDAL_EXPORT
    infer_ops_dispatcher<dal::detail::host_policy, double, method::lloyd_dense, task::clustering>;

}  // namespace oneapi::dal::kmeans::detail::v1
