// The reference's benchmark driver (mpi/main.cc:34-178, graph500_bfs) on one
// GPU: generate, construct, find_roots, run_bfs per root with validation, and
// the Graph500 result block.  Usage:
//
//   g500_main SCALE [EDGEFACTOR] [--roots N] [--reorder 0|1|2] [--max-runs K]
//             [--pre-exec SECONDS] [--autotune]
//   g500_main --print-result LOGFILE_PATH
//
// --print-result prints the result block of the runs a resume file holds,
// without a GPU (the statistics of print_bfs_result, logfile.h:49-107).
//
// LOGFILE=path resumes an interrupted run as the reference does
// (benchmark_helper.hpp:530-604): the file keeps SCALE, edgefactor, the
// generation/construction times and every finished root's (BFS time,
// validation time, edge count); a rerun with the same parameters starts at
// the first unfinished root, a mismatching file is an error.  --max-runs K
// stops after K roots of this invocation (for interrupted runs on purpose).
// The BFS time of a root is the host wall time of run_bfs with pred in host
// memory, as main.cc:115-117 takes it.
#include <algorithm>
#include <chrono>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "g500_bfs.hpp"

namespace {

// LogFileFormat (logfile.h:109-124): same fields and layout, so that resume
// files keep their meaning.
struct LogFileTime {
  double bfs_time;
  double validate_time;
  int64_t edge_counts;
};
struct LogFileFormat {
  int scale;
  int edge_factor;
  int mpi_size;
  int num_runs;
  double generation_time;
  double construction_time;
  double redistribution_time;
  LogFileTime times[64];
};

// Order statistics of the Graph500 output (the specification's definitions:
// quartiles as the mean of the two middle order statistics, sample stddev).
struct Stats {
  double min, q1, median, q3, max, mean, stddev;
};

Stats statistics(std::vector<double> x) {
  Stats s{};
  const size_t n = x.size();
  if (n == 0) return s;
  double sum = 0;
  for (double v : x) sum += v;
  s.mean = sum / (double)n;
  double var = 0;
  for (double v : x) var += (v - s.mean) * (v - s.mean);
  s.stddev = n > 1 ? std::sqrt(var / (double)(n - 1)) : 0.0;
  std::sort(x.begin(), x.end());
  s.min = x[0];
  s.q1 = (x[(n - 1) / 4] + x[n / 4]) * .5;
  s.median = (x[(n - 1) / 2] + x[n / 2]) * .5;
  s.q3 = (x[n - 1 - (n - 1) / 4] + x[n - 1 - n / 4]) * .5;
  s.max = x[n - 1];
  return s;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void print_result(int scale, int edgefactor, int nroots, double gen, double cons, const std::vector<double>& bfs,
                  const std::vector<double>& val, const std::vector<double>& edges, bool ok) {
  std::printf("============= Result ==============\n");
  std::printf("SCALE:                          %d\n", scale);
  std::printf("edgefactor:                     %d\n", edgefactor);
  std::printf("NBFS:                           %d\n", nroots);
  std::printf("graph_generation:               %g\n", gen);
  std::printf("num_mpi_processes:              %d\n", 1);
  std::printf("construction_time:              %g\n", cons);
  std::printf("redistribution_time:            %g\n", 0.0);
  if (!ok) {
    std::printf("No results printed for invalid run.\n");
    return;
  }
  Stats t = statistics(bfs);
  std::printf("min_time:                       %.12g\n", t.min);
  std::printf("firstquartile_time:             %.12g\n", t.q1);
  std::printf("median_time:                    %.12g\n", t.median);
  std::printf("thirdquartile_time:             %.12g\n", t.q3);
  std::printf("max_time:                       %.12g\n", t.max);
  std::printf("mean_time:                      %.12g\n", t.mean);
  std::printf("stddev_time:                    %.12g\n", t.stddev);
  Stats e = statistics(edges);
  std::printf("min_nedge:                      %.11g\n", e.min);
  std::printf("firstquartile_nedge:            %.11g\n", e.q1);
  std::printf("median_nedge:                   %.11g\n", e.median);
  std::printf("thirdquartile_nedge:            %.11g\n", e.q3);
  std::printf("max_nedge:                      %.11g\n", e.max);
  std::printf("mean_nedge:                     %.11g\n", e.mean);
  std::printf("stddev_nedge:                   %.11g\n", e.stddev);
  std::vector<double> spe(bfs.size());
  for (size_t i = 0; i < bfs.size(); ++i) spe[i] = bfs[i] / edges[i];
  Stats r = statistics(spe);
  std::printf("min_TEPS:                       %.12g\n", 1. / r.max);
  std::printf("firstquartile_TEPS:             %.12g\n", 1. / r.q3);
  std::printf("median_TEPS:                    %.12g\n", 1. / r.median);
  std::printf("thirdquartile_TEPS:             %.12g\n", 1. / r.q1);
  std::printf("max_TEPS:                       %.12g\n", 1. / r.min);
  std::printf("harmonic_mean_TEPS:             %.12g\n", 1. / r.mean);
  // standard error of the harmonic mean (Norris 1940), as the specification gives it
  std::printf("harmonic_stddev_TEPS:           %.12g\n",
              r.stddev / (r.mean * r.mean * std::sqrt((double)std::max<size_t>(spe.size(), 2) - 1)));
  Stats v = statistics(val);
  std::printf("min_validate:                   %.12g\n", v.min);
  std::printf("firstquartile_validate:         %.12g\n", v.q1);
  std::printf("median_validate:                %.12g\n", v.median);
  std::printf("thirdquartile_validate:         %.12g\n", v.q3);
  std::printf("max_validate:                   %.12g\n", v.max);
  std::printf("mean_validate:                  %.12g\n", v.mean);
  std::printf("stddev_validate:                %.12g\n", v.stddev);
}

void usage() {
  std::fprintf(stderr,
               "usage: g500_main SCALE [EDGEFACTOR] [--roots N] [--reorder 0|1|2] [--max-runs K] "
               "[--pre-exec SECONDS] [--autotune]\n"
               "       g500_main --print-result LOGFILE_PATH\n");
}

// The result block of the finished runs of a resume file.
int print_log_result(const char* path) {
  LogFileFormat log;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) {
    std::fprintf(stderr, "cannot open %s\n", path);
    return 1;
  }
  const size_t got = std::fread(&log, sizeof(log), 1, fp);
  std::fclose(fp);
  if (got != 1 || log.num_runs < 1 || log.num_runs > 64) {
    std::fprintf(stderr, "%s is not a log file with finished runs\n", path);
    return 1;
  }
  std::vector<double> bfs, val, edges;
  for (int i = 0; i < log.num_runs; ++i) {
    bfs.push_back(log.times[i].bfs_time);
    val.push_back(log.times[i].validate_time);
    edges.push_back((double)log.times[i].edge_counts);
  }
  print_result(log.scale, log.edge_factor, log.num_runs, log.generation_time, log.construction_time, bfs, val, edges,
               true);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  int scale = -1, edgefactor = 16, nroots = 64, reorder = 2, max_runs = -1;
  double pre_exec = 0;
  bool tune = false;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--help" || a == "-h") {
      usage();
      return 0;
    } else if (a == "--print-result" && i + 1 < argc) {
      return print_log_result(argv[i + 1]);
    } else if (a == "--roots" && i + 1 < argc) {
      nroots = std::atoi(argv[++i]);
    } else if (a == "--reorder" && i + 1 < argc) {
      reorder = std::atoi(argv[++i]);
    } else if (a == "--max-runs" && i + 1 < argc) {
      max_runs = std::atoi(argv[++i]);
    } else if (a == "--pre-exec" && i + 1 < argc) {
      pre_exec = std::atof(argv[++i]);
    } else if (a == "--autotune") {
      tune = true;
    } else if (scale < 0) {
      scale = std::atoi(a.c_str());
    } else {
      edgefactor = std::atoi(a.c_str());
    }
  }
  if (scale < 1 || scale > 36 || edgefactor < 1 || nroots < 1 || nroots > 64 || reorder < 0 || reorder > 2) {
    usage();
    return 2;
  }
  try {
    std::vector<double> bfs_times(64, 0), validate_times(64, 0), edge_counts(64, 0);
    LogFileFormat log;
    std::memset(&log, 0, sizeof(log));
    int root_start = 0;
    const char* logname = std::getenv("LOGFILE");
    if (logname) {  // read_log_file (benchmark_helper.hpp:530-573)
      if (FILE* fp = std::fopen(logname, "rb")) {
        const size_t got = std::fread(&log, sizeof(log), 1, fp);
        std::fclose(fp);
        if (got != 1 || log.scale != scale || log.edge_factor != edgefactor || log.mpi_size != 1 ||
            log.num_runs < 0 || log.num_runs > 64) {
          std::fprintf(stderr, "Log file is not match the current run: params:(current),(log): SCALE:%d,%d, "
                               "edgefactor:%d,%d, size:%d,%d\n",
                       scale, log.scale, edgefactor, log.edge_factor, 1, log.mpi_size);
          return 1;
        }
        root_start = log.num_runs;
        std::printf("===== LOG START =====\n");
        std::printf("graph_generation:               %f s\n", log.generation_time);
        std::printf("construction_time:              %f s\n", log.construction_time);
        for (int i = 0; i < root_start; ++i) {
          std::printf("Time for BFS %d is %f\n", i, log.times[i].bfs_time);
          std::printf("Validate time for BFS %d is %f\n", i, log.times[i].validate_time);
          std::printf("TEPS for BFS %d is %g\n", i, (double)log.times[i].edge_counts / log.times[i].bfs_time);
          bfs_times[i] = log.times[i].bfs_time;
          validate_times[i] = log.times[i].validate_time;
          edge_counts[i] = (double)log.times[i].edge_counts;
        }
        std::printf("=====  LOG END  =====\n");
        if (root_start) std::printf("Resume from %d th run\n", root_start);
      }
    }

    g500cpp::BfsOnGPU bench(reorder);
    bench.generate_and_construct(scale, edgefactor);
    double generation_time = 0, construction_time = 0;
    g500cpp::check(g500_graph_timings(bench.graph_.handle(), &generation_time, &construction_time));
    std::vector<int64_t> roots((size_t)nroots);
    int found = nroots;
    g500cpp::find_roots(bench.graph_, roots.data(), found);
    nroots = found;
    const int64_t nlocalverts = bench.graph_.pred_size();
    int64_t* pred = nullptr;
    g500cpp::check(g500_host_alloc(sizeof(int64_t) * (uint64_t)nlocalverts, reinterpret_cast<void**>(&pred)));
    if (root_start == 0) {  // init_log (benchmark_helper.hpp:595-604)
      log.scale = scale;
      log.edge_factor = edgefactor;
      log.mpi_size = 1;
      log.generation_time = generation_time;
      log.construction_time = construction_time;
      log.redistribution_time = 0;
      log.num_runs = 0;
    }
    bench.prepare_bfs();
    if (tune) {
      const g500_tune_result r = bench.autotune(roots.data(), std::min(nroots, 8));
      std::printf("autotune: policy %d alpha %g beta %g (%d settings)\n", r.policy, r.alpha, r.beta, r.configs_tried);
    }
    for (double left = pre_exec; left > 0;) {  // PRE_EXEC_TIME warm-up (main.cc:91-103)
      const double t = now_s();
      bench.run_bfs(roots[0], pred);
      left -= now_s() - t;
    }
    bool ok = true;
    int done_now = 0;
    for (int i = root_start; i < nroots; ++i) {
      if (max_runs >= 0 && done_now >= max_runs) break;
      std::printf("========== Running BFS %d ==========\n", i);
      double t = now_s();
      bench.run_bfs(roots[(size_t)i], pred);
      bfs_times[(size_t)i] = now_s() - t;
      bench.get_pred(pred);
      std::printf("Time for BFS %d is %f\n", i, bfs_times[(size_t)i]);
      t = now_s();
      int64_t evc = 0;
      ok = g500cpp::validate_bfs_result(bench.graph_, roots[(size_t)i], pred, &evc);
      validate_times[(size_t)i] = now_s() - t;
      edge_counts[(size_t)i] = (double)evc;
      std::printf("Validate time for BFS %d is %f\n", i, validate_times[(size_t)i]);
      std::printf("Number of traversed edges is %" PRId64 "\n", evc);
      std::printf("TEPS for BFS %d is %g\n", i, (double)evc / bfs_times[(size_t)i]);
      if (!ok) break;
      ++done_now;
      if (logname) {  // update_log_file (benchmark_helper.hpp:575-593)
        LogFileTime& lt = log.times[log.num_runs++];
        lt.bfs_time = bfs_times[(size_t)i];
        lt.validate_time = validate_times[(size_t)i];
        lt.edge_counts = evc;
        if (FILE* fp = std::fopen(logname, "wb")) {
          std::fwrite(&log, sizeof(log), 1, fp);
          std::fclose(fp);
        } else {
          std::fprintf(stderr, "Cannot create log file ... skipping\n");
        }
      }
    }
    bench.end_bfs();
    g500_host_free(pred);
    const int finished = root_start + done_now;
    if (finished < nroots && ok) {
      std::printf("stopped after %d of %d roots (--max-runs); rerun with the same LOGFILE to resume\n", finished,
                  nroots);
      return 0;
    }
    bfs_times.resize((size_t)nroots);
    validate_times.resize((size_t)nroots);
    edge_counts.resize((size_t)nroots);
    print_result(scale, edgefactor, nroots, log.generation_time, log.construction_time, bfs_times, validate_times,
                 edge_counts, ok);
    return ok ? 0 : 3;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}
