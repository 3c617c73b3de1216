// cucm_decompress -- drop-in for the reference's decompressor CLI
// (main, cucm_decompress_v2.cu:1258-1314): -i, -o, -a.  -a sets the
// speculation depth as the reference does (it decodes up to a+1 bits per
// step); it changes speed only, never the output.
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>

#include "../../include/cucm.h"
#include "cli_common.h"

static void print_help(const char *prog) {
  std::cout << "Usage: " << prog << " -i <input_file> -o <output_file> [-a <maxassumed_length>]\n"
            << "  -i <input_file>        Input compressed file\n"
            << "  -o <output_file>       Output decompressed file\n"
            << "  -a <N>                 Speculate N+1 bits per decode step (default: 3)\n"
            << "  -d <ID>                CUDA device (default: 0)\n";
}

int main(int argc, char **argv) {
  const char *in_path = nullptr, *out_path = nullptr;
  int a = 3, device = 0;
  for (int i = 1; i < argc; i++) {
    if (std::strcmp(argv[i], "-i") == 0 && i + 1 < argc) in_path = argv[++i];
    else if (std::strcmp(argv[i], "-o") == 0 && i + 1 < argc) out_path = argv[++i];
    else if (std::strcmp(argv[i], "-a") == 0 && i + 1 < argc) a = std::atoi(argv[++i]);
    else if (std::strcmp(argv[i], "-d") == 0 && i + 1 < argc) device = std::atoi(argv[++i]);
    else {
      print_help(argv[0]);
      return 1;
    }
  }
  if (!in_path || !out_path) {
    print_help(argv[0]);
    return 1;
  }
  std::vector<uint8_t> data;
  if (!cucm_cli::read_file(in_path, data)) {
    std::cerr << "Error: cannot open input file " << in_path << "\n";
    return 1;
  }
  uint64_t size = 0;
  if (cucm_decompressed_size(data.data(), data.size(), &size)) {
    std::cerr << "Error: not a CuCM container\n";
    return 1;
  }
  auto t0 = std::chrono::high_resolution_clock::now();
  cucm_tuning tu;
  std::memset(&tu, 0, sizeof tu);
  tu.spec_bits = a + 1 < 1 ? 1 : (a + 1 > 8 ? 8 : a + 1);
  cucm_ctx *ctx = nullptr;
  int rc = cucm_ctx_create(device, &tu, &ctx);
  if (rc) {
    std::cerr << "cucm: " << cucm_strerror(rc) << std::endl;
    return 1;
  }
  std::vector<uint8_t> out(size ? size : 1);
  uint64_t out_n = 0;
  rc = cucm_decompress(ctx, data.data(), data.size(), out.data(), out.size(), &out_n);
  double dev_ms = 0;
  cucm_last_device_ms(ctx, &dev_ms);
  cucm_ctx_destroy(ctx);
  if (rc) {
    std::cerr << "cucm: " << cucm_strerror(rc) << std::endl;
    return 1;
  }
  if (!cucm_cli::write_file(out_path, out.data(), out_n)) {
    std::cerr << "Error: cannot open output file " << out_path << "\n";
    return 1;
  }
  auto t1 = std::chrono::high_resolution_clock::now();
  std::cout << "Decompression finished: " << in_path << " -> " << out_path << " (" << out_n
            << " bytes, maxassumed_length=" << a << ")\n";
  std::cout << "Device time: " << dev_ms / 1000.0 << " sec" << std::endl;
  std::cout << "Total time: " << std::chrono::duration<double>(t1 - t0).count() << " sec" << std::endl;
  return 0;
}
