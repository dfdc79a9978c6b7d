// epik2_v4 -- command-line drop-in for the reference's GPU programs.
//
//   epik2_v4 <num_samples> <num_snps> [block_size]        (GPU/v4.cpp:210-212; v1-v3 take
//                                                          the first two arguments only)
//   epik2_v4 --file <geno.bin> <num_samples> <num_snps>   (matrix + phenotype from a file:
//                                                          n*m genotype bytes, sample-major,
//                                                          then n phenotype bytes)
//   epik2_v4 --plink <prefix> [missing_genotype]          (PLINK 1 binary fileset
//                                                          <prefix>.bed/.bim/.fam; missing
//                                                          genotypes read as the given value,
//                                                          default 0)
//
// With positional arguments the data is the reference's own synthetic input
// (srand(100) generator, GPU/v4.cpp:81-110) and the output has the reference's lines
// (GPU/v4.cpp:251, 610-612):
//   Selected device: <name>
//   Time: <seconds>
//   Score: <K2 score>
//   Solution: <i> <j> <k>
// `block_size` only tiled the reference's launches; the search here needs no tiling, so
// the value is checked (positive) and otherwise unused.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/epik2.h"

static int usage(const char* argv0) {
  std::fprintf(stderr,
               "usage: %s <num_samples> <num_snps> [block_size]\n"
               "       %s --file <geno.bin> <num_samples> <num_snps>\n"
               "       %s --plink <prefix> [missing_genotype]\n",
               argv0, argv0, argv0);
  return 2;
}

int main(int argc, char** argv) {
  if (argc < 3) return usage(argv[0]);
  long long n = 0, m = 0;
  std::vector<uint8_t> geno, pheno;
  if (std::strcmp(argv[1], "--plink") == 0) {
    int64_t ns = 0, ms = 0;
    int r = epik2_plink_dims(argv[2], &ns, &ms);
    if (r != EPIK2_OK || ns < 1 || ms < 3) {
      std::fprintf(stderr, "cannot read PLINK fileset %s: %s\n", argv[2], epik2_strerror(r ? r : EPIK2_E_INVALID));
      return 1;
    }
    n = ns;
    m = ms;
    geno.resize((size_t)(n * m));
    pheno.resize((size_t)n);
    const int missing = argc > 3 ? std::atoi(argv[3]) : 0;
    r = epik2_read_plink(argv[2], (uint8_t)missing, geno.data(), pheno.data());
    if (r != EPIK2_OK) {
      std::fprintf(stderr, "cannot read PLINK fileset %s: %s\n", argv[2], epik2_strerror(r));
      return 1;
    }
  } else if (std::strcmp(argv[1], "--file") == 0) {
    if (argc < 5) return usage(argv[0]);
    n = std::atoll(argv[3]);
    m = std::atoll(argv[4]);
    if (n < 1 || m < 3) return usage(argv[0]);
    geno.resize((size_t)(n * m));
    pheno.resize((size_t)n);
    FILE* f = std::fopen(argv[2], "rb");
    if (!f) {
      std::fprintf(stderr, "cannot open %s\n", argv[2]);
      return 1;
    }
    size_t got = std::fread(geno.data(), 1, geno.size(), f);
    got += std::fread(pheno.data(), 1, pheno.size(), f);
    std::fclose(f);
    if (got != geno.size() + pheno.size()) {
      std::fprintf(stderr, "short read from %s\n", argv[2]);
      return 1;
    }
  } else {
    n = std::atoll(argv[1]);
    m = std::atoll(argv[2]);
    if (n < 1 || m < 3) return usage(argv[0]);
    if (argc > 3 && std::atoll(argv[3]) < 1) return usage(argv[0]);
    geno.resize((size_t)(n * m));
    pheno.resize((size_t)n);
    if (epik2_generate_reference(n, m, geno.data(), pheno.data()) != EPIK2_OK) return usage(argv[0]);
  }

  epik2_ctx* ctx = nullptr;
  int r = epik2_create(&ctx, 0);
  if (r != EPIK2_OK) {
    std::fprintf(stderr, "epik2: %s\n", epik2_strerror(r));
    return 1;
  }
  char name[256];
  epik2_device_name(ctx, name, sizeof(name));
  std::cout << "Selected device: " << name << std::endl;
  int32_t id = 0;
  r = epik2_load_u8(ctx, geno.data(), pheno.data(), n, m, &id);
  if (r != EPIK2_OK) {
    std::fprintf(stderr, "epik2: %s: %s\n", epik2_strerror(r), epik2_last_error(ctx));
    epik2_destroy(ctx);
    return 1;
  }
  epik2_best best{};
  auto t0 = std::chrono::steady_clock::now();
  r = epik2_scan(ctx, id, nullptr, &best);
  auto t1 = std::chrono::steady_clock::now();
  if (r != EPIK2_OK) {
    std::fprintf(stderr, "epik2: %s: %s\n", epik2_strerror(r), epik2_last_error(ctx));
    epik2_destroy(ctx);
    return 1;
  }
  std::cout << "Time: " << std::chrono::duration<double>(t1 - t0).count() << std::endl;
  std::cout << "Score: " << best.score << std::endl;
  std::cout << "Solution: " << best.i << " " << best.j << " " << best.k << std::endl;
  epik2_destroy(ctx);
  return 0;
}
