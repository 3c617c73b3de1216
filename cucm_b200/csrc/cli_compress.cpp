// cucm_compress -- drop-in for the reference's compressor CLI
// (main, cucm_compress_v2.cu:1301-1418): same flags, same defaults, same
// container on disk.
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/cucm.h"
#include "cli_common.h"

static void print_help(const char *prog) {
  std::cout << "Usage: " << prog << " [options]\n"
            << "Options:\n"
            << "  -c, --chunknum <N>    Number of chunks (default: file_size/chunksize + 1)\n"
            << "  -s, --chunksize <SZ>  Size of each chunk, supports K/M/G suffix (default: 1M)\n"
            << "  -u, --unit <SZ>       Unit size in bits, multiple of 32 up to 1024 (default: 128)\n"
            << "  -f, --file <path>     Input file to compress (default: ./enwik8)\n"
            << "  -o, --output <path>   Output compressed file (default: ./compressed.bin)\n"
            << "  -p, --prelearn <SZ>   Prelearn size, supports K/M/G suffix (default: 0 = disabled)\n"
            << "  -b, --batch <NUM>     Chunks per container batch (default: 100)\n"
            << "  -F, --fixed           Fixed-model variant: code with the prelearned model, no updates\n"
            << "                        (needs -p; not a reference stream)\n"
            << "  -d, --device <ID>     CUDA device (default: 0)\n"
            << "  -h, --help            Show this help message\n";
}

int main(int argc, char **argv) {
  if (argc == 1) {
    print_help(argv[0]);
    return 0;
  }
  cucm_params p;
  cucm_default_params(&p);
  long chunknum = -1;
  int unit = 128, batch = 100, device = 0;
  std::string in_path = "./enwik8", out_path = "./compressed.bin";
  for (int i = 1; i < argc; i++) {
    auto is = [&](const char *a, const char *b) {
      return (std::strcmp(argv[i], a) == 0 || std::strcmp(argv[i], b) == 0) && i + 1 < argc;
    };
    if (is("-c", "--chunknum")) {
      chunknum = std::atol(argv[++i]);
      if (chunknum <= 0) {
        std::cerr << "Invalid chunknum: " << chunknum << std::endl;
        return 1;
      }
    } else if (is("-s", "--chunksize")) {
      p.chunksize = cucm_cli::parse_size(argv[++i]);
      if (p.chunksize == 0) {
        std::cerr << "Invalid chunk size: " << argv[i] << std::endl;
        return 1;
      }
    } else if (is("-f", "--file")) {
      in_path = argv[++i];
    } else if (is("-o", "--output")) {
      out_path = argv[++i];
    } else if (is("-p", "--prelearn")) {
      p.prelearn = cucm_cli::parse_size(argv[++i]);
      if (p.prelearn == 0) std::cerr << "Warning: prelearn disabled (size=0)" << std::endl;
    } else if (is("-u", "--unit")) {
      unit = std::atoi(argv[++i]);
      if (unit <= 0 || unit % 32 != 0 || unit > 1024) {
        std::cerr << "Invalid unit size: " << unit << " (must be a multiple of 32, at most 1024)" << std::endl;
        return 1;
      }
    } else if (is("-b", "--batch")) {
      batch = std::atoi(argv[++i]);
      if (batch <= 0 || batch > 65535) {
        std::cerr << "Invalid batch number: " << batch << std::endl;
        return 1;
      }
    } else if (std::strcmp(argv[i], "-F") == 0 || std::strcmp(argv[i], "--fixed") == 0) {
      p.fixed_model = 1;
    } else if (is("-d", "--device")) {
      device = std::atoi(argv[++i]);
    } else if (std::strcmp(argv[i], "-h") == 0 || std::strcmp(argv[i], "--help") == 0) {
      print_help(argv[0]);
      return 0;
    } else {
      std::cerr << "Unknown option: " << argv[i] << std::endl;
      print_help(argv[0]);
      return 1;
    }
  }
  p.unit = (uint32_t)unit;
  p.batch = (uint32_t)batch;
  if (p.fixed_model && p.prelearn == 0) {
    std::cerr << "The fixed-model variant (-F) needs a prelearn prefix (-p)" << std::endl;
    return 1;
  }
  std::vector<uint8_t> data;
  if (!cucm_cli::read_file(in_path.c_str(), data)) {
    std::cerr << "Failed to open input file: " << in_path << std::endl;
    return 1;
  }
  uint64_t n = data.size();
  if (chunknum > 0 && p.chunksize * (uint64_t)chunknum < n) n = p.chunksize * (uint64_t)chunknum;  // -c truncates
  if (p.prelearn > n) {
    std::cerr << "Invalid prelearn size: " << p.prelearn << " exceeds the input (" << n << " bytes)" << std::endl;
    return 1;
  }
  std::cout << "Compressing file: " << in_path << ", filesize: " << n << ", chunksize: " << p.chunksize
            << ", unit: " << p.unit << ", prelearn: " << p.prelearn << ", batch: " << p.batch
            << ", output: " << out_path << std::endl;
  auto t0 = std::chrono::high_resolution_clock::now();
  cucm_ctx *ctx = nullptr;
  int rc = cucm_ctx_create(device, nullptr, &ctx);
  if (rc) {
    std::cerr << "cucm: " << cucm_strerror(rc) << std::endl;
    return 1;
  }
  std::vector<uint8_t> out(cucm_compress_bound(n, &p));
  uint64_t out_n = 0;
  rc = cucm_compress(ctx, data.data(), n, &p, out.data(), out.size(), &out_n);
  double dev_ms = 0;
  cucm_last_device_ms(ctx, &dev_ms);
  cucm_ctx_destroy(ctx);
  if (rc) {
    std::cerr << "cucm: " << cucm_strerror(rc) << std::endl;
    return 1;
  }
  if (!cucm_cli::write_file(out_path.c_str(), out.data(), out_n)) {
    std::cerr << "Failed to open output file: " << out_path << std::endl;
    return 1;
  }
  auto t1 = std::chrono::high_resolution_clock::now();
  uint64_t nchunks = n > p.prelearn ? (n - p.prelearn + p.chunksize - 1) / p.chunksize : 0;
  uint64_t nbatches = (nchunks + p.batch - 1) / p.batch;
  // the reference's count leaves out the batch size fields (8 bytes each in
  // the 64-bit container, which inputs past 4 GiB get)
  uint64_t reported = out_n - (n > 0xffffffffull ? 8 : 4) * nbatches;
  std::cout << "Original size  : " << n << " bytes\n";
  std::cout << "Compressed size: " << reported << " bytes\n";
  std::cout << "Compression ratio: " << (reported ? (double)n / (double)reported : 0.0) << "\n";
  std::cout << "Device time: " << dev_ms / 1000.0 << " sec" << std::endl;
  std::cout << "Total time: " << std::chrono::duration<double>(t1 - t0).count() << " sec" << std::endl;
  return 0;
}
