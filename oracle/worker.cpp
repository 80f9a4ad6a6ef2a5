// Oracle worker speaking the reference benchmark-worker protocol
// (benchmark-tools/worker/src/main.rs:14-49): argv LOG2 READY_PATH PROOF_PATH;
// write READY after setup; read the decimal seed from stdin; prove; write
// PROOF.tmp and rename.  Test infrastructure (see flockref.hpp): it lets the
// reference's trusted verifier check the oracle's proofs end to end.
#include "flockref.hpp"
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

using namespace flockref;

int main(int argc, char** argv) {
  // optional 4th argument: a directory where (seed, proof) pairs are recorded
  // before publication, so a fixture script can pin verifier-accepted bytes
  if (argc != 4 && argc != 5) {
    fprintf(stderr, "usage: flockref_worker LOG2 READY_PATH PROOF_PATH [RECORD_DIR]\n");
    return 2;
  }
  int log2 = atoi(argv[1]);
  if (log2 < 8 || log2 > 20) return 2;
  blake3_r1cs(log2);  // setup: matrices + statement digest
  ligerito_config(14 + log2);
  FILE* rf = fopen(argv[2], "wb");
  if (!rf) return 1;
  fputs("ready\n", rf);
  fclose(rf);
  std::string line;
  if (!std::getline(std::cin, line)) return 1;
  uint64_t seed = std::stoull(line);
  auto blocks = generate_compressions((uint32_t)log2, seed);
  Bundle b = prove(blocks, log2, "flock-bench-v0");
  std::vector<uint8_t> bytes = serialize(b);
  if (argc == 5) {
    std::string rec = std::string(argv[4]) + "/proof_" + std::to_string(log2) + "_" + std::to_string(seed) + ".bin";
    FILE* rfp = fopen(rec.c_str(), "wb");
    if (rfp) {
      fwrite(bytes.data(), 1, bytes.size(), rfp);
      fclose(rfp);
    }
  }
  std::string tmp = std::string(argv[3]) + ".tmp";
  FILE* pf = fopen(tmp.c_str(), "wb");
  if (!pf) return 1;
  fwrite(bytes.data(), 1, bytes.size(), pf);
  fclose(pf);
  if (rename(tmp.c_str(), argv[3]) != 0) return 1;
  return 0;
}
