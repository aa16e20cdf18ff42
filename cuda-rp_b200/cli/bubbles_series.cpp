// `bubbles_series NAME`: the reference's sweep script scripts/executor.sh NAME
// (:1-47) as one native program.  For every configuration file
// CONFS/NAME_<i>.txt, in the order `ls` lists them, it copies the file into
// RESULTS/<date>/<HH:MM>/ and runs it as `bubbles` runs a file, with
// RESULTS/<date>/<HH:MM>/rawdata_<i>/ as the target directory.  The runs share
// the GPU: each simulation has its own CUDA stream and is driven from a pool of
// host threads, largest cells x steps first, so that small grids that cannot
// fill the GPU alone overlap.  Each run's output is what `bubbles -d
// rawdata_<i>/ NAME_<i>.txt` writes (rawdata, tracker files, *_minmax.txt,
// runtime.txt).
//
//   bubbles_series [-h] [-a] [-s] [--confs DIR] [--results DIR] [--threads N] [--dry-run] NAME
//
// Not part of it: the gnuplot step (scripts/plot_results_child.sh) and the copy
// of plot.gnu.  The script passes the target directory as a second positional
// argument, which the reference's parser does not take (its input-file option
// holds one value, src/bubbles.cpp:135,146); here the directory is used as the
// target, the evident intent.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <ctime>
#include <filesystem>
#include <iostream>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "crp.h"
#include "run_conf.h"

namespace fs = std::filesystem;

namespace {

const char* kHelp =
    "Usage: bubbles_series [options] NAME\n\n"
    "Runs every CONFS/NAME_<i>.txt as `bubbles` would, into RESULTS/<date>/<HH:MM>/rawdata_<i>/,\n"
    "the simulations concurrently on one GPU.\n\n"
    "  -h [ --help ]          Output this help message.\n"
    "  -a [ --ascii ]         Save plaintext files (as bubbles -a).\n"
    "  -s [ --sph ]           Save sph files (as bubbles -s).\n"
    "  --confs DIR            Directory of the configuration files (default: confs).\n"
    "  --results DIR          Results directory (default: results).\n"
    "  --threads N            Simulations in flight at once (default: all, at most 16).\n"
    "  --dry-run              Print the plan; create and run nothing.\n";

struct Job {
  std::string number;  // <i> of NAME_<i>.txt
  std::string conf;    // path of the configuration file
  double work = 0.0;   // cells x steps, for the order (0 when the file does not parse)
};

std::string local_time(time_t now, const char* fmt) {
  struct tm t;
  localtime_r(&now, &t);
  char buf[64];
  strftime(buf, sizeof(buf), fmt, &t);
  return buf;
}

// mkdir with the script's messages (executor.sh:8-24).
bool make_dir(const fs::path& d, const char* exists_word, std::ostream& out) {
  std::error_code ec;
  if (fs::is_directory(d, ec)) {
    out << d.string() << " " << exists_word << std::endl;
    return true;
  }
  fs::create_directory(d, ec);
  if (ec) {
    std::cerr << "error: cannot create " << d.string() << ": " << ec.message() << std::endl;
    return false;
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  std::string name, confs = "confs", results = "results";
  bool ascii = false, sph = false, dry = false;
  int threads = 0;
  for (int k = 1; k < argc; k++) {
    const std::string a = argv[k];
    auto value = [&](const char* opt) -> const char* {
      if (k + 1 >= argc) {
        std::cerr << "the required argument for option '" << opt << "' is missing" << std::endl;
        std::exit(1);
      }
      return argv[++k];
    };
    if (a == "-h" || a == "--help") {
      std::cout << kHelp << std::endl;
      return 0;
    } else if (a == "-a" || a == "--ascii") {
      ascii = true;
    } else if (a == "-s" || a == "--sph") {
      sph = true;
    } else if (a == "--confs") {
      confs = value("--confs");
    } else if (a == "--results") {
      results = value("--results");
    } else if (a == "--threads") {
      threads = std::atoi(value("--threads"));
    } else if (a == "--dry-run") {
      dry = true;
    } else if (!a.empty() && a[0] == '-') {
      std::cerr << "unknown option " << a << std::endl;
      return 1;
    } else if (name.empty()) {
      name = a;
    }
  }
  if (name.empty()) {
    std::cout << "Please specify the name of a configuration series" << std::endl;
    return 1;
  }
  // ls CONFS/NAME_*.txt (executor.sh:3): <i> is what the glob's * matched.
  std::vector<Job> jobs;
  std::error_code ec;
  const std::string pre = name + "_";
  for (const auto& e : fs::directory_iterator(confs, ec)) {
    const std::string f = e.path().filename().string();
    if (f.size() >= pre.size() + 4 && f.compare(0, pre.size(), pre) == 0 && f.compare(f.size() - 4, 4, ".txt") == 0)
      jobs.push_back(Job{f.substr(pre.size(), f.size() - pre.size() - 4), e.path().string(), 0.0});
  }
  if (ec || jobs.empty()) {
    std::cerr << "error: no configuration file " << confs << "/" << pre << "*.txt" << std::endl;
    return 1;
  }
  std::sort(jobs.begin(), jobs.end(), [](const Job& x, const Job& y) { return x.conf < y.conf; });
  for (Job& j : jobs) {
    crp_config c;
    crp_config_defaults(&c);
    if (crp_config_parse_file(j.conf.c_str(), &c, nullptr, 0) == CRP_OK)
      j.work = (double)c.grid_x * (double)c.grid_y * (double)std::max(c.sim_n_step_max, 1);
  }
  const time_t now = time(nullptr);
  const fs::path day = fs::path(results) / local_time(now, "%Y-%m-%d");
  const fs::path run_dir = day / local_time(now, "%H:%M");
  if (dry) {
    std::cout << "results: " << run_dir.string() << std::endl;
    for (const Job& j : jobs)
      std::cout << j.conf << " -> " << (run_dir / ("rawdata_" + j.number)).string() << "/" << std::endl;
    return 0;
  }
  if (!make_dir(results, "exists", std::cout) || !make_dir(day, "exists", std::cout) ||
      !make_dir(run_dir, "exits", std::cout))
    return 1;
  for (const Job& j : jobs) {
    fs::copy_file(j.conf, run_dir / (pre + j.number + ".txt"), fs::copy_options::overwrite_existing, ec);
    if (ec) {
      std::cerr << "error: cannot copy " << j.conf << ": " << ec.message() << std::endl;
      return 1;
    }
  }
  // Largest cells x steps first; each thread takes the next file when its run ends.
  std::vector<size_t> order(jobs.size());
  for (size_t k = 0; k < order.size(); k++) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return jobs[x].work > jobs[y].work; });
  const int n_threads = std::max(1, std::min<int>(threads > 0 ? threads : 16, (int)jobs.size()));
  std::atomic<size_t> next{0};
  std::mutex io;
  std::vector<int> status(jobs.size(), 0);
  auto worker = [&]() {
    for (;;) {
      const size_t q = next.fetch_add(1);
      if (q >= order.size()) return;
      const Job& j = jobs[order[q]];
      {
        std::lock_guard<std::mutex> g(io);
        std::cout << std::endl << "Processing " << pre << j.number << ".txt" << std::endl << std::endl;
      }
      ConfRun run;
      run.in_file = j.conf;
      run.target_dir = (run_dir / ("rawdata_" + j.number)).string() + "/";
      run.ascii = ascii;
      run.sph = sph;
      run.dir_given = true;
      run.progress = false;
      std::ostringstream out, err;
      status[order[q]] = run_configuration(run, out, err);
      std::lock_guard<std::mutex> g(io);
      std::cout << "[" << pre << j.number << ".txt] " << out.str() << std::flush;
      if (!err.str().empty()) std::cerr << "[" << pre << j.number << ".txt] " << err.str() << std::flush;
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < n_threads; t++) pool.emplace_back(worker);
  for (std::thread& t : pool) t.join();
  int failed = 0;
  for (size_t k = 0; k < jobs.size(); k++) failed += status[k] != 0;
  if (failed) std::cerr << failed << " of " << jobs.size() << " configurations failed" << std::endl;
  return failed ? 1 : 0;
}
