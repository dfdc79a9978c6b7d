// Input formats and result statistics around the search (include/epik2.h, "Input files"
// and "Permutation tests").  Host C++ only; no device code.
//
// PLINK 1 binary fileset: <prefix>.fam (one line per sample, whitespace-separated; column 6
// is the phenotype: 2 = case, 1 = control, anything else = missing), <prefix>.bim (one line
// per SNP) and <prefix>.bed (magic 0x6c 0x1b, mode 0x01 = SNP-major; per SNP ceil(N/4) bytes,
// sample s in bits 2(s%4)..2(s%4)+1 of byte s/4; 00 = homozygous first allele, 10 =
// heterozygous, 11 = homozygous second allele, 01 = missing).  The search's genotype is the
// count of the first allele (00 -> 2, 10 -> 1, 11 -> 0); samples with a missing phenotype are
// left out; missing genotypes take the caller's value.
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/epik2.h"

namespace {

// phenotype per .fam line: 1 case, 0 control, -1 missing
int read_fam(const std::string& path, std::vector<int8_t>* status) {
  std::ifstream f(path);
  if (!f) return EPIK2_E_NOT_FOUND;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream ls(line);
    std::string col[6];
    int n = 0;
    while (n < 6 && (ls >> col[n])) n++;
    if (n == 0) continue;  // blank line
    if (n < 6) return EPIK2_E_INVALID;
    status->push_back(col[5] == "2" ? 1 : (col[5] == "1" ? 0 : -1));
  }
  return EPIK2_OK;
}

int count_lines(const std::string& path, int64_t* n) {
  std::ifstream f(path);
  if (!f) return EPIK2_E_NOT_FOUND;
  std::string line;
  *n = 0;
  while (std::getline(f, line)) {
    for (char c : line)
      if (!std::isspace((unsigned char)c)) {
        (*n)++;
        break;
      }
  }
  return EPIK2_OK;
}

}  // namespace

extern "C" {

int epik2_plink_dims(const char* prefix, int64_t* n_samples, int64_t* n_snps) {
  if (!prefix || !n_samples || !n_snps) return EPIK2_E_INVALID;
  std::vector<int8_t> status;
  int r = read_fam(std::string(prefix) + ".fam", &status);
  if (r) return r;
  int64_t m = 0;
  r = count_lines(std::string(prefix) + ".bim", &m);
  if (r) return r;
  int64_t n = 0;
  for (int8_t s : status) n += s >= 0;
  *n_samples = n;
  *n_snps = m;
  return EPIK2_OK;
}

int epik2_read_plink(const char* prefix, uint8_t missing_genotype, uint8_t* geno, uint8_t* pheno) {
  if (!prefix || !geno || !pheno) return EPIK2_E_INVALID;
  std::vector<int8_t> status;
  int r = read_fam(std::string(prefix) + ".fam", &status);
  if (r) return r;
  int64_t m = 0;
  r = count_lines(std::string(prefix) + ".bim", &m);
  if (r) return r;
  const int64_t n_all = (int64_t)status.size();
  std::vector<int64_t> keep;  // .fam rows with a phenotype, in file order
  for (int64_t s = 0; s < n_all; s++)
    if (status[(size_t)s] >= 0) keep.push_back(s);
  const int64_t n = (int64_t)keep.size();
  FILE* f = std::fopen((std::string(prefix) + ".bed").c_str(), "rb");
  if (!f) return EPIK2_E_NOT_FOUND;
  unsigned char magic[3];
  if (std::fread(magic, 1, 3, f) != 3 || magic[0] != 0x6c || magic[1] != 0x1b || magic[2] != 0x01) {
    std::fclose(f);
    return EPIK2_E_INVALID;  // not a SNP-major .bed
  }
  const int64_t row = (n_all + 3) / 4;
  std::vector<unsigned char> buf((size_t)row);
  static const uint8_t code[4] = {2, 0, 1, 0};  // 00, 01 (missing: replaced below), 10, 11
  for (int64_t j = 0; j < m; j++) {
    if ((int64_t)std::fread(buf.data(), 1, (size_t)row, f) != row) {
      std::fclose(f);
      return EPIK2_E_INVALID;  // truncated
    }
    for (int64_t t = 0; t < n; t++) {
      const int64_t s = keep[(size_t)t];
      const unsigned v = (buf[(size_t)(s >> 2)] >> (2 * (s & 3))) & 3u;
      geno[t * m + j] = v == 1 ? missing_genotype : code[v];
    }
  }
  std::fclose(f);
  for (int64_t t = 0; t < n; t++) pheno[t] = (uint8_t)status[(size_t)keep[(size_t)t]];
  return EPIK2_OK;
}

double epik2_perm_pvalue(float observed, const float* replicate_best, int64_t n_replicates) {
  if (n_replicates < 0 || (n_replicates > 0 && !replicate_best)) return -1.0;
  int64_t as_good = 0;
  for (int64_t r = 0; r < n_replicates; r++) as_good += replicate_best[r] <= observed;
  return (double)(1 + as_good) / (double)(1 + n_replicates);
}

}  // extern "C"
