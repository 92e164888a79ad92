// A oneDAL client written only against the unchanged oneDAL public headers
// (oneapi/dal/algo/kmeans.hpp, oneapi/dal/table/homogen.hpp): dal::train and
// dal::infer on the gold known-answer data of the reference test suite
// (cpp/oneapi/dal/algo/kmeans/test/data.hpp), read from a text file. Linked
// against the B200 dispatchers, every call below runs on the GPU.
//
//   kmeans_client <gold.txt> <float|double>
// prints: iterations, objective, centroids, responses, infer objective, then the
// smoke case of the reference suite (fixture.hpp:221-252) trained WITHOUT initial
// centroids (oneDAL's default k-means++ init): smoke_centroids, smoke_responses.
//
//   kmeans_client serialize <centroids.txt> <float|double> <out.bin>
// builds kmeans::model from "k d v..." (k = 0: a default model without centroids)
// and writes oneDAL's binary archive of it (detail::serialize into
// binary_output_archive, cpp/oneapi/dal/detail/archives.hpp). No GPU is used.
//
//   kmeans_client deserialize <in.bin> <float|double>
// reads such an archive with oneDAL's binary_input_archive + detail::deserialize
// and prints: cluster_count, centroids (or "exception: <what>").
#include "oneapi/dal/algo/kmeans.hpp"
#include "oneapi/dal/detail/archives.hpp"
#include "oneapi/dal/detail/serialization.hpp"
#include "oneapi/dal/table/csr.hpp"
#include "oneapi/dal/table/homogen.hpp"
#include "oneapi/dal/table/row_accessor.hpp"

#include <cstdio>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

namespace dal = oneapi::dal;

template <typename F>
int run(const std::vector<double> &xs, std::int64_t n, std::int64_t d, const std::vector<double> &cs,
        std::int64_t k) {
    std::vector<F> x(xs.begin(), xs.end()), c(cs.begin(), cs.end());
    const auto data = dal::homogen_table::wrap(x.data(), n, d);
    const auto init = dal::homogen_table::wrap(c.data(), k, d);
    const auto desc = dal::kmeans::descriptor<F>().set_cluster_count(k).set_max_iteration_count(100).set_accuracy_threshold(0.0);
    const auto result = dal::train(desc, data, init);
    std::printf("iterations %lld\n", (long long)result.get_iteration_count());
    std::printf("objective %.10g\n", result.get_objective_function_value());
    const auto cen = dal::row_accessor<const F>(result.get_model().get_centroids()).pull({ 0, -1 });
    std::printf("centroids");
    for (std::int64_t i = 0; i < cen.get_count(); ++i) std::printf(" %.9g", (double)cen[i]);
    std::printf("\n");
    const auto desc_inf = dal::kmeans::descriptor<F>().set_cluster_count(k).set_result_options(
        dal::kmeans::result_options::compute_exact_objective_function);
    const auto inf = dal::infer(desc_inf, result.get_model(), data);
    const auto lab = dal::row_accessor<const std::int32_t>(inf.get_responses()).pull({ 0, -1 });
    std::printf("responses");
    for (std::int64_t i = 0; i < lab.get_count(); ++i) std::printf(" %d", lab[i]);
    std::printf("\n");
    std::printf("infer_objective %.10g\n", inf.get_objective_function_value());
    // a precondition the reference checks before dispatch (detail/train_ops.hpp:50-52)
    try {
        dal::train(dal::kmeans::descriptor<F>().set_cluster_count(n + 1), data, dal::homogen_table{});
        std::printf("precondition not enforced\n");
    } catch (const dal::invalid_argument &) {
        std::printf("invalid_argument ok\n");
    }
    const F smoke[] = { 1, 1, 2, 2, 1, 2, 2, 1, -1, -1, -1, -2, -2, -1, -2, -2 };
    const auto smoke_data = dal::homogen_table::wrap(smoke, 8, 2);
    const auto smoke_res = dal::train(
        dal::kmeans::descriptor<F>().set_cluster_count(2).set_max_iteration_count(4).set_accuracy_threshold(0.001),
        smoke_data);
    const auto sc = dal::row_accessor<const F>(smoke_res.get_model().get_centroids()).pull({ 0, -1 });
    std::printf("smoke_centroids");
    for (std::int64_t i = 0; i < sc.get_count(); ++i) std::printf(" %.9g", (double)sc[i]);
    std::printf("\n");
    const auto sr = dal::row_accessor<const std::int32_t>(smoke_res.get_responses()).pull({ 0, -1 });
    std::printf("smoke_responses");
    for (std::int64_t i = 0; i < sr.get_count(); ++i) std::printf(" %d", sr[i]);
    std::printf("\n");
    // 'KMeans CSR exact objective accounts for unstored features' (test/batch.cpp:406-480)
    // through dal::train / dal::infer on a one-based csr_table
    const F cv[] = { 10, 10, 20 };
    const std::int64_t ci[] = { 1, 2, 3 }, ro[] = { 1, 2, 3, 4 };
    const F cinit[] = { 5, 5, 0, 0, 0, 20 };
    const auto csr = dal::csr_table::wrap(cv, ci, ro, 3, 3, dal::sparse_indexing::one_based);
    const auto csr_desc = dal::kmeans::descriptor<F, dal::kmeans::method::lloyd_csr>()
                              .set_cluster_count(2)
                              .set_max_iteration_count(1)
                              .set_accuracy_threshold(0.0)
                              .set_result_options(dal::kmeans::result_options::compute_exact_objective_function);
    const auto csr_res = dal::train(csr_desc, csr, dal::homogen_table::wrap(cinit, 2, 3));
    const auto crr = dal::row_accessor<const std::int32_t>(csr_res.get_responses()).pull({ 0, -1 });
    std::printf("csr_responses");
    for (std::int64_t i = 0; i < crr.get_count(); ++i) std::printf(" %d", crr[i]);
    std::printf("\n");
    std::printf("csr_objective %.10g\n", csr_res.get_objective_function_value());
    const auto csr_inf = dal::infer(csr_desc, csr_res.get_model(), csr);
    std::printf("csr_infer_objective %.10g\n", csr_inf.get_objective_function_value());
    return 0;
}

template <typename F>
int serialize_model(const char *in, const char *out) {
    std::ifstream f(in);
    std::int64_t k, d;
    f >> k >> d;
    std::vector<F> c(k * d);
    for (auto &v : c) {
        double x;
        f >> x;
        v = F(x);
    }
    dal::kmeans::model<> m;
    if (k > 0) m.set_centroids(dal::homogen_table::wrap(c.data(), k, d));
    dal::detail::binary_output_archive ar;
    dal::detail::serialize(m, ar);
    const auto bytes = ar.to_array();
    std::FILE *o = std::fopen(out, "wb");
    if (!o) return 1;
    std::fwrite(bytes.get_data(), 1, bytes.get_count(), o);
    std::fclose(o);
    std::printf("bytes %lld\n", (long long)bytes.get_count());
    return 0;
}

template <typename F>
int deserialize_model(const char *in) {
    std::ifstream f(in, std::ios::binary);
    const std::vector<char> raw((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    dal::detail::binary_input_archive ar(reinterpret_cast<const dal::byte_t *>(raw.data()),
                                         (std::int64_t)raw.size());
    dal::kmeans::model<> m;
    dal::detail::deserialize(m, ar);
    std::printf("cluster_count %lld\n", (long long)m.get_cluster_count());
    std::printf("centroids");
    if (m.get_cluster_count() > 0) {
        const auto c = dal::row_accessor<const F>(m.get_centroids()).pull({ 0, -1 });
        for (std::int64_t i = 0; i < c.get_count(); ++i) std::printf(" %.17g", (double)c[i]);
    }
    std::printf("\n");
    return 0;
}

int main(int argc, char **argv) {
    if (argc >= 5 && std::string(argv[1]) == "serialize") {
        try {
            return std::string(argv[3]) == "double" ? serialize_model<double>(argv[2], argv[4])
                                                    : serialize_model<float>(argv[2], argv[4]);
        } catch (const std::exception &e) {
            std::printf("exception: %s\n", e.what());
            return 1;
        }
    }
    if (argc >= 4 && std::string(argv[1]) == "deserialize") {
        try {
            return std::string(argv[3]) == "double" ? deserialize_model<double>(argv[2])
                                                    : deserialize_model<float>(argv[2]);
        } catch (const std::exception &e) {
            std::printf("exception: %s\n", e.what());
            return 1;
        }
    }
    if (argc < 3) return 2;
    std::ifstream f(argv[1]);
    std::int64_t n, d, k;
    f >> n >> d >> k;
    std::vector<double> x(n * d), c(k * d);
    for (auto &v : x) f >> v;
    for (auto &v : c) f >> v;
    const std::string t = argv[2];
    try {
        return t == "double" ? run<double>(x, n, d, c, k) : run<float>(x, n, d, c, k);
    } catch (const std::exception &e) {
        std::printf("exception: %s\n", e.what());
        return 1;
    }
}
