// flock_worker: the B200 prover behind the reference benchmark-worker process
// protocol (benchmark-tools/worker/src/main.rs:14-49, harness worker_command
// benchmark-tools/harness/src/main.rs:215-352):
//   flock_worker LOG2 READY_PATH PROOF_PATH [RECORD_DIR]
// Untimed: context, setup for 2^LOG2 compressions and one warm-up proof, then
// READY_PATH is created.  Timed: read the decimal seed from stdin, prove the
// benchmark inputs of that seed, write PROOF_PATH.tmp and rename it to
// PROOF_PATH.  Uses only the C ABI of libflockgpu.so.
// With RECORD_DIR (not part of the reference protocol; a wrapper script adds
// it), the proof is also written to RECORD_DIR/proof_<LOG2>_<seed>.bin before
// it is published, so a harness run leaves (seed, proof) pairs behind.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>
#include "../../include/flock_gpu.h"

namespace {
const char kDomain[] = "flock-bench-v0";  // benchmark-tools/common/src/lib.rs:2

int fail(flock_ctx* ctx, const char* what, int rc) {
  fprintf(stderr, "flock_worker: %s failed (%d): %s\n", what, rc, ctx ? flock_last_error(ctx) : "");
  return 1;
}
}  // namespace

int main(int argc, char** argv) {
  if (argc != 4 && argc != 5) {
    fprintf(stderr, "usage: flock_worker LOG2 READY_PATH PROOF_PATH [RECORD_DIR]\n");
    return 2;
  }
  const int log2 = atoi(argv[1]);
  if (log2 < 8 || log2 > 20) {
    fprintf(stderr, "flock_worker: LOG2 must be in 8..=20\n");
    return 2;
  }
  flock_ctx* ctx = nullptr;
  int rc = flock_ctx_create(0, 0, &ctx);
  if (rc) return fail(ctx, "flock_ctx_create", rc);
  flock_setup* setup = nullptr;
  rc = flock_setup_create(ctx, (uint32_t)log2, FLOCK_HASH_BLAKE3, FLOCK_PROFILE_FAST, &setup);
  if (rc) return fail(ctx, "flock_setup_create", rc);
  std::vector<uint8_t> proof(500000);
  size_t len = 0;
  const uint8_t* dom = reinterpret_cast<const uint8_t*>(kDomain);
  rc = flock_prove_seed(setup, 0x00C0FFEEBEEFD15Cull, dom, strlen(kDomain), proof.data(), proof.size(), &len);
  if (rc) return fail(ctx, "warm-up proof", rc);
  FILE* rf = fopen(argv[2], "wb");
  if (!rf) return fail(ctx, "creating READY_PATH", 0);
  fputs("ready\n", rf);
  fclose(rf);

  std::string line;
  if (!std::getline(std::cin, line)) return fail(ctx, "reading the seed", 0);
  const uint64_t seed = std::stoull(line);
  rc = flock_prove_seed(setup, seed, dom, strlen(kDomain), proof.data(), proof.size(), &len);
  if (rc) return fail(ctx, "proof", rc);
  if (argc == 5) {
    const std::string rec = std::string(argv[4]) + "/proof_" + std::to_string(log2) + "_" + std::to_string(seed) + ".bin";
    FILE* f = fopen(rec.c_str(), "wb");
    if (!f || fwrite(proof.data(), 1, len, f) != len) return fail(ctx, "writing the record", 0);
    fclose(f);
  }
  const std::string tmp = std::string(argv[3]) + ".tmp";
  FILE* pf = fopen(tmp.c_str(), "wb");
  if (!pf || fwrite(proof.data(), 1, len, pf) != len) return fail(ctx, "writing PROOF_PATH.tmp", 0);
  fclose(pf);
  if (rename(tmp.c_str(), argv[3]) != 0) return fail(ctx, "publishing PROOF_PATH", 0);
  flock_setup_destroy(setup);
  flock_ctx_destroy(ctx);
  return 0;
}
