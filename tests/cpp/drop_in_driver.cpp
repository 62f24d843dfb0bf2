// Drop-in check: the reference carousel driver's call sequence
// (src/CPRA_MKL.cpp:35-140, ShrinkWrap_CPRA_MKL_Sample) issued through the
// abstract interface CPRA::CpraImpl<float>* on a B200Impl<float>, with buffers
// in managed memory that the host fills and reads like the reference's main()
// (src/CPRA_MKL.cpp:156-232, include/detail/CPRA.inl:8-28).
//
//   drop_in_driver <in_dir> <out_file>
// in_dir holds cfg.txt ("M N L P B epi iter preit beta"), A.f32 / S.f32
// ([P][M][N] float32) and x0.c64 ([P][B][M][N] complex64); out_file receives
// x ([P][B][M][N] complex64) followed by the P*B convergence errors (float32).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>

#include "cpra_b200/B200_Impl.hpp"

using C = std::complex<float>;

namespace {

bool read_file(const std::string& path, void* dst, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    const size_t got = std::fread(dst, 1, bytes, f);
    std::fclose(f);
    return got == bytes;
}

void dm_iteration(CPRA::CpraImpl<float>* impl, C* x, C* t1, C* t2, float* A, float* S, uint64_t num, uint64_t B,
                  float Beta) {
    impl->Forward2D(t1);
    impl->DataConstraint(t1, A, num, B);
    impl->Backward2D(t1);
    impl->MergeAddData(x, t1, -1.0 / Beta, 1.0 + 1.0 / Beta, num);
    impl->SpaceConstraint(t1, S, num, B);
    impl->SpaceConstraint(t2, S, num, B);
    impl->MergeAddData(x, t2, 1.0 / Beta, 1.0 - 1.0 / Beta, num);
    impl->Forward2D(t2);
    impl->DataConstraint(t2, A, num, B);
    impl->Backward2D(t2);
    impl->MergeAddData(t1, x, Beta, 1.0, num);
    impl->MergeAddData(t2, x, -1.0 * Beta, 1.0, num);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <in_dir> <out_file>\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    unsigned long long M, N, L, P, B;
    int epi, iter, preit;
    float Beta;
    FILE* cf = std::fopen((dir + "/cfg.txt").c_str(), "r");
    if (!cf || std::fscanf(cf, "%llu %llu %llu %llu %llu %d %d %d %f", &M, &N, &L, &P, &B, &epi, &iter, &preit,
                           &Beta) != 9) {
        std::fprintf(stderr, "bad cfg.txt\n");
        return 2;
    }
    std::fclose(cf);
    auto owner = std::make_unique<CPRA::B200Impl<float>>(M, N, L, B);
    CPRA::B200Impl<float>* b200 = owner.get();
    CPRA::CpraImpl<float>* impl = b200;  // everything below sees only the interface
    const uint64_t MNB = M * N * B;
    auto* A = static_cast<float*>(b200->Allocate(sizeof(float) * M * N * P));
    auto* S = static_cast<float*>(b200->Allocate(sizeof(float) * M * N * P));
    auto* x = static_cast<C*>(b200->Allocate(sizeof(C) * MNB * P));
    auto* t1 = static_cast<C*>(b200->Allocate(sizeof(C) * MNB));
    auto* t2 = static_cast<C*>(b200->Allocate(sizeof(C) * MNB));
    auto* old = static_cast<C*>(b200->Allocate(sizeof(C) * MNB));
    auto* err = static_cast<float*>(b200->Allocate(sizeof(float) * P * B));
    if (!read_file(dir + "/A.f32", A, sizeof(float) * M * N * P) || !read_file(dir + "/S.f32", S, sizeof(float) * M * N * P) ||
        !read_file(dir + "/x0.c64", x, sizeof(C) * MNB * P)) {
        std::fprintf(stderr, "cannot read inputs\n");
        return 2;
    }
    std::memset(err, 0, sizeof(float) * P * B);
    const size_t bytes = sizeof(C) * MNB;
    // Step A (:35-56)
    impl->Memcpy(t1, x, bytes);
    impl->Memcpy(t2, x, bytes);
    for (int i = 0; i < preit; ++i) dm_iteration(impl, x, t1, t2, A, S, MNB, B, Beta);
    impl->Sync();
    // Step B (:59-124)
    for (int e = 0; e < epi; ++e) {
        for (uint64_t p = 0; p < P; ++p) {
            C* xp = x + MNB * p;
            if (p == P - 1) {
                impl->MergeAddData(x + MNB * (p - 1), xp, 0.5, 0.5, MNB);
            } else if (p == 0) {
                impl->MergeAddData(x + MNB * (p + 1), xp, 0.5, 0.5, MNB);
            } else {
                impl->MergeAddData(x + MNB * (p - 1), xp, 0.5, 0, MNB);
                impl->MergeAddData(x + MNB * (p + 1), xp, 0.5, 1, MNB);
            }
            impl->Memcpy(t1, xp, bytes);
            impl->Memcpy(t2, xp, bytes);
            for (int i = 0; i < iter; ++i) {
                const bool last = (i == iter - 1 && e == epi - 1);
                if (last) impl->Memcpy(old, xp, bytes);
                dm_iteration(impl, xp, t1, t2, A + M * N * p, S + M * N * p, MNB, B, Beta);
                if (last) {
                    impl->Memcpy(t1, xp, bytes);
                    impl->Forward2D(old);
                    impl->Forward2D(t1);
                    impl->ConvergeError(old, t1, err + B * p, M, N, 1, B);
                }
            }
        }
    }
    // final projection (:126-140)
    for (uint64_t p = 0; p < P; ++p) {
        C* xp = x + MNB * p;
        impl->Memcpy(t1, xp, bytes);
        impl->Forward2D(t1);
        impl->DataConstraint(t1, A + M * N * p, MNB, B);
        impl->Backward2D(t1);
        impl->MergeAddData(xp, t1, -1.0 / Beta, 1.0 + 1.0 / Beta, MNB);
        impl->SpaceConstraint(t1, S + M * N * p, MNB, B);
        impl->Memcpy(xp, t1, bytes);
    }
    impl->Sync();
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    std::fwrite(x, sizeof(C), MNB * P, out);  // the host reads managed memory directly
    std::fwrite(err, sizeof(float), P * B, out);
    std::fclose(out);
    for (void* p : {(void*)A, (void*)S, (void*)x, (void*)t1, (void*)t2, (void*)old, (void*)err}) b200->Deallocate(p);
    return 0;
}
