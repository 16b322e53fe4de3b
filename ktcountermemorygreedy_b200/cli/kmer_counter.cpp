// kmer_counter -- drop-in for the reference counter's command line
// (src/main.cpp:481-633):
//   kmer_counter <fastq|dir|a,b,...> <k_len> <n_thread> <memory_limit_gb> <temp_dir>
//                [map_capacity] [filter_min=2] [filter_max=4294967295] [count_max=255]
// It counts on the GPU through libkc and writes temp_dir/infos.bin, high.bin
// (exact counts) and an empty low.bin, which the reference's histogram_tool
// and dump_tool read unchanged.  n_thread and map_capacity are validated as
// the reference does and otherwise unused (the device schedules itself).
// KC_BLOOM=1 in the environment runs the reference's Bloom singleton split.
#include <cerrno>
#include <chrono>
#include <iostream>

#include "cli_common.h"

static int usage(const char *p)
{
    std::cerr << "Usage: " << p
              << " <fastq_file> <k_len> <n_thread> <memory_limit_gb> <temp_dir> [map_capacity] [filter_min=2] "
                 "[filter_max=4294967295] [count_max=255]"
              << std::endl;
    return 1;
}

int main(int argc, char **argv)
{
    if (argc < 6 || argc > 10) return usage(argv[0]);
    uint32_t k = 0, n_thread = 0, map_cap = 1024, fmin = 2, fmax = 0xffffffffu, cmax = 255;
    uint64_t mem_gb = 0;
    if (!cli::parse_u32(argv[2], k) || !cli::parse_u32(argv[3], n_thread) || !cli::parse_u64(argv[4], mem_gb))
        return usage(argv[0]);
    if (argc >= 7 && !cli::parse_u32(argv[6], map_cap)) return usage(argv[0]);
    if (argc >= 8 && !cli::parse_u32(argv[7], fmin)) return usage(argv[0]);
    if (argc >= 9 && !cli::parse_u32(argv[8], fmax)) return usage(argv[0]);
    if (argc >= 10 && !cli::parse_u32(argv[9], cmax)) return usage(argv[0]);
    if (n_thread < 6) {
        std::cerr << "n_thread must be >= 6" << std::endl;
        return 255;
    }
    // rounded up to a power of two, at least 1024, below 16M (src/main.cpp:541, :581)
    uint64_t map_pow2 = 1;
    while (map_pow2 < map_cap) map_pow2 <<= 1;
    map_pow2 = std::max<uint64_t>(1024, map_pow2);
    if (map_pow2 >= 16ull * 1024 * 1024 || fmax < fmin || cmax == 0) return usage(argv[0]);
    if (k == 0 || k > 128) {
        std::cerr << "k_len must be <= 128" << std::endl;
        return 1;
    }
    const std::string tmp = cli::with_slash(argv[5]);
    // infos.bin first, before any input is read (src/main.cpp:588-595)
    {
        FILE *f = std::fopen((tmp + "infos.bin").c_str(), "wb");
        if (!f) {
            std::cerr << "Open infos.bin failed : " << std::strerror(errno) << std::endl;
            return 1;
        }
        const uint32_t info[2] = {k, cmax};
        const bool ok = std::fwrite(info, sizeof(info), 1, f) == 1;
        if ((std::fclose(f) != 0) || !ok) {
            std::cerr << "Write infos.bin failed" << std::endl;
            return 1;
        }
    }
    auto names = cli::input_files(argv[1]);
    if (names.empty()) {
        std::cerr << "No input files" << std::endl;
        return 255;
    }
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::vector<char>> data(names.size());
    std::vector<kc_buffer> files(names.size());
    for (size_t i = 0; i < names.size(); ++i) {
        if (!cli::read_file(names[i], data[i])) {
            std::cerr << "Failed to open: " << names[i] << std::endl;
            return 255;
        }
        files[i] = kc_buffer{data[i].data(), data[i].size()};
    }
    kc_handle *h = nullptr;
    kc_config cfg{};
    if (kc_open(&cfg, &h) != KC_OK) {
        std::cerr << "kc_open: " << kc_last_error() << std::endl;
        return 2;
    }
    kc_job job;
    kc_job_defaults(&job);
    job.files = files.data();
    job.n_files = (uint32_t)files.size();
    job.k = k;
    job.count_max = cmax;
    job.memory_gb = mem_gb ? mem_gb : 1;
    job.filter_min = fmin;
    job.filter_max = fmax;
    const char *bl = std::getenv("KC_BLOOM");
    job.bloom = (bl && bl[0] == '1') ? 1 : 0;
    // high.bin is packed on the device; the records themselves stay there
    job.pack_high = 1;
    job.keep_records = 0;
    kc_job_id id = 0;
    int rc = kc_submit(h, &job, &id);
    if (rc == KC_OK) rc = kc_wait(h, id, -1);
    if (rc == KC_OK) rc = kc_write_tmpdir(h, id, tmp.c_str());
    kc_result_t r{};
    if (rc == KC_OK) rc = kc_result(h, id, &r);
    if (rc != KC_OK) {
        std::cerr << "kmer_counter: " << kc_last_error() << std::endl;
        kc_close(h);
        return 2;
    }
    auto us = std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "Total read k-mer count: " << r.occurrences << std::endl;
    std::cout << "Total elapsed us: " << us << std::endl;
    std::cout << "High frequency unique k-mer : " << r.n_records_total << std::endl;
    kc_close(h);
    return 0;
}
