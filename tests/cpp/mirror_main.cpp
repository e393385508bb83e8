// Drives the C++ mirror (include/mlods.hpp) the way scene::projectPoints and
// scene::projectPointsOnCPU drive the reference classes: build the octree,
// upload queries, project in place one iteration per call, read back; and
// projectCPU per query.  Reads points/normals/queries from raw float files and
// writes the projections for the test to compare.
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <thread>
#include <vector>

#include "mlods.hpp"

using mlods::vec3;

static std::vector<vec3> read_vec3(const char* path)
{
    std::vector<vec3> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) std::exit(2);
    vec3 x;
    while (std::fread(&x, sizeof x, 1, f) == 1) v.push_back(x);
    std::fclose(f);
    return v;
}

static void write_vec3(const char* path, const std::vector<vec3>& v)
{
    FILE* f = std::fopen(path, "wb");
    std::fwrite(v.data(), sizeof(vec3), v.size(), f);
    std::fclose(f);
}

int main(int argc, char** argv)
{
    if (argc < 7) return 1;  // pts nrm queries out_gpu out_cpu sigma_rel
    const std::vector<vec3> pts = read_vec3(argv[1]), nrm = read_vec3(argv[2]);
    std::vector<vec3> q = read_vec3(argv[3]);
    const float sigma_rel = float(std::atof(argv[6]));
    auto* tree = new mlods::APSSOctree();
    tree->build(pts, nrm);
    mlods::Kernel k;
    k.type = mlods::Kernel::GAUSSIAN;
    k.sigma = sigma_rel;
    k.updateSigmas(true, tree->getBoundingBox().radius());  // scene::setNewKernel scales by the box radius
    mlods::Fastapss apss(tree, k, unsigned(q.size()));
    apss.setScalingProtectionSphere(3.f);
    apss.copyPointsToGPU(unsigned(q.size()), q.data());
    std::vector<vec3> out(q.size()), outn(q.size());
    for (int tick = 0; tick < 10; ++tick) apss.project(unsigned(q.size()), nullptr, nullptr, 1, k);
    apss.project(unsigned(q.size()), out.data(), outn.data(), 0, k);
    write_vec3(argv[4], out);
    std::vector<vec3> cpu(q.size()), cpun(q.size());
    for (size_t i = 0; i < q.size(); ++i) apss.projectCPU(q[i], cpu[i], cpun[i], 10, k);
    write_vec3(argv[5], cpu);
    // the same calls from 16 host threads at once, interleaved over the
    // queries as an OpenMP static schedule with chunk 1 would deal them
    // (scene.cpp:982-986): results must equal the serial ones bit for bit
    std::vector<vec3> par(q.size()), parn(q.size());
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < 16; ++t)
            pool.emplace_back([&, t] {
                for (size_t i = size_t(t); i < q.size(); i += 16) apss.projectCPU(q[i], par[i], parn[i], 10, k);
            });
        for (std::thread& th : pool) th.join();
    }
    for (size_t i = 0; i < q.size(); ++i)
        if (par[i].x != cpu[i].x || par[i].y != cpu[i].y || par[i].z != cpu[i].z || parn[i].x != cpun[i].x ||
            parn[i].y != cpun[i].y || parn[i].z != cpun[i].z) {
            std::fprintf(stderr, "threaded projectCPU differs from the serial result at query %zu\n", i);
            return 4;
        }
    // the walk schedule tuned on the queries, then the same ten project calls:
    // any schedule agrees with one query per warp to float rounding
    const int chosen = apss.tuneSchedule(unsigned(q.size()), q.data(), 10);
    if (chosen != 1 && chosen != 2 && chosen != 4) return 5;
    apss.queries_per_warp = 2;
    apss.copyPointsToGPU(unsigned(q.size()), q.data());
    for (int tick = 0; tick < 10; ++tick) apss.project(unsigned(q.size()), nullptr, nullptr, 1, k);
    std::vector<vec3> out2(q.size()), out2n(q.size());
    apss.project(unsigned(q.size()), out2.data(), out2n.data(), 0, k);
    const float r = tree->getBoundingBox().radius();
    for (size_t i = 0; i < q.size(); ++i) {
        const float dx = out2[i].x - out[i].x, dy = out2[i].y - out[i].y, dz = out2[i].z - out[i].z;
        if (std::sqrt(dx * dx + dy * dy + dz * dz) > 2e-5f * r) {  // 1e-5 of the diagonal
            std::fprintf(stderr, "two queries per warp differ from one at query %zu\n", i);
            return 6;
        }
    }
    if (argc > 7) {  // APSSOctree::cpuSphere at the queries: u0, u123, u4 per query
        std::vector<float> u;
        for (const vec3& x : q) {
            float u0 = 0.f, u4 = 0.f;
            vec3 u123(0.f, 0.f, 0.f);
            tree->cpuSphere(x, u0, u123, u4, k);
            u.insert(u.end(), {u0, u123.x, u123.y, u123.z, u4});
        }
        FILE* f = std::fopen(argv[7], "wb");
        if (!f) return 2;
        std::fwrite(u.data(), sizeof(float), u.size(), f);
        std::fclose(f);
        std::vector<vec3> nb;
        tree->getKnn(q[0], 8, nb);
        if (nb.size() != 8) return 3;
    }
    std::printf("nodes %u depth %u\n", tree->nbOfNodes(), tree->computeDepth());
    delete tree;
    return 0;
}
