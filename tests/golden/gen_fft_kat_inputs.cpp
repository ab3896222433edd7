// Regenerates the seeded inputs of the reference's FFNT known-answer tests
// (test/test_fft_roundtrip.cu:145-149 and :249-253) with the same standard
// library engines and distributions:
//   fft_roundtrip_in.f64     1024 doubles, std::mt19937(42),
//                            uniform_real_distribution<double>(-100, 100)
//   negacyclic_random_in.i32 1024 ints,    std::mt19937(123),
//                            uniform_int_distribution<int>(-5, 5)
#include <cstdio>
#include <random>
#include <vector>

int main(int argc, char** argv)
{
    const char* dir = argc > 1 ? argv[1] : ".";
    char path[4096];
    {
        std::mt19937 rng(42);
        std::uniform_real_distribution<double> dist(-100.0, 100.0);
        std::vector<double> v(1024);
        for (auto& x : v) x = dist(rng);
        std::snprintf(path, sizeof(path), "%s/fft_roundtrip_in.f64", dir);
        FILE* f = std::fopen(path, "wb");
        std::fwrite(v.data(), sizeof(double), v.size(), f);
        std::fclose(f);
    }
    {
        std::mt19937 rng(123);
        std::uniform_int_distribution<int> dist(-5, 5);
        std::vector<int> v(1024);
        for (auto& x : v) x = dist(rng);
        std::snprintf(path, sizeof(path), "%s/negacyclic_random_in.i32", dir);
        FILE* f = std::fopen(path, "wb");
        std::fwrite(v.data(), sizeof(int), v.size(), f);
        std::fclose(f);
    }
    return 0;
}
