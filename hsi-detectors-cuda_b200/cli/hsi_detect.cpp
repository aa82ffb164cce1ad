// hsi_detect - target detection over a stream of hyperspectral frames.
//
// The reference's command-line consumer (src/main.cpp:19-292) on this
// library: the same flags, defaults and report, and the same exit codes
// (0 done, 1 a setup or run failure, 2 a usage error).  Added flags:
//   --detector=sam|cem|rx|ace  the detector that is scored and thresholded.
//                              SAM streams through hsi::Pipeline as in the
//                              reference; CEM, RX and ACE run per frame on
//                              the frame's own statistics (hsi::
//                              DeviceStatistics, launch_cem / launch_rx_ace,
//                              launch_detect)
//   --batch                    the --frames frames as one batch through the
//                              batch runner (include/hsi_batch.h), captured
//                              as a CUDA graph and replayed --repeat times;
//                              its lists are SAM, ACE and RX
//   --repeat=N                 timed replays of the batch
//   --pfa=RATE                 RX false-alarm rate; the RX threshold is the
//                              chi-square quantile at this rate unless
//                              --threshold is given
//   --loading=F                diagonal loading of the statistics
//   --autotune                 time the batch runner's choices on the batch
//   --lagged                   CEM, RX or ACE with lagged statistics (include/
//                              hsi_lagged.h): frame k is scored with frame
//                              k-1's statistics while its own are built on a
//                              second stream; the RX threshold comes from --pfa
// Flags are checked before the device is touched, so a usage error exits 2
// on any machine.  Sources: synthetic, and ENVI replay (--envi, --resident);
// the HOT snapshot-mosaic directory source is not built and exits 2.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "hsi/detect_cuda.hpp"
#include "hsi/detector.hpp"
#include "hsi/detectors.hpp"
#include "hsi/frame_source.hpp"
#include "hsi/pipeline.hpp"
#include "hsi/sam_cuda.hpp"
#include "hsi/spectra_io.hpp"
#include "hsi_batch.h"
#include "hsi_lagged.h"

namespace {

const char* kUsage = R"(hsi_detect - hyperspectral target detection (SAM, CEM, RX, ACE) on the GPU

  hsi_detect [options]

Source
  --source=synthetic|envi       where frames come from            [synthetic]
                                (hot is not built here)
  --envi=A.hdr,B.hdr            ENVI cubes to replay
  --resident=N                  cubes held in RAM                         [4]
  --width=N --height=N          synthetic frame size               [512x512]
  --bands=N                     synthetic band count                    [128]
  --targets=N                   synthetic planted targets                 [3]
  --noise=F                     synthetic noise sigma                  [0.01]

Detection
  --detector=sam|cem|rx|ace     detector scored and thresholded         [sam]
  --library=FILE.csv            target spectra; required unless the source
                                supplies its own (--source=synthetic does)
  --threshold=X                 SAM angle (rad) [0.10]; CEM response [0.5];
                                ACE score [0.5]; RX: from --pfa
  --pfa=RATE                    RX false-alarm rate                    [1e-4]
  --loading=F                   diagonal loading of the statistics     [1e-6]
  --nms=N                       non-maximum suppression radius, 0 off      [2]
  --max-detections=N            detection list capacity                [4096]

Execution
  --variant=baseline|optimized|half                              [optimized]
  --memory=copy|zerocopy        zerocopy is rejected: the scorer streams the
                                cube from device memory
  --streams=N                   frames in flight (SAM)                     [3]
  --frames=N                    frames to process                        [300]
  --warmup=N                    unmeasured frames first                   [30]
  --prefill                     stage the ring once and replay it (SAM)
  --batch                       score --frames frames as one batch (SAM, ACE
                                or RX lists), replayed as a CUDA graph
  --repeat=N                    timed replays of the batch                [10]
  --autotune                    time the batch runner's choices first
  --lagged                      CEM/RX/ACE: score each frame with the previous
                                frame's statistics, built on a second stream
  --csv=FILE                    write per-frame timings
  --print-detections=N          print the first N detections of the last frame
  --dump-score=FILE             write the last frame's score map as raw float32
                                (height*width, raster order)
  --quiet
  --help)";

struct Args {
  std::map<std::string, std::string> values;

  bool has(const std::string& key) const { return values.count(key) != 0; }
  std::string str(const std::string& key, const std::string& fallback) const {
    const auto it = values.find(key);
    return (it == values.end() || it->second.empty()) ? fallback : it->second;
  }
};

// --key=value and --key tokens; anything else is ignored, as the reference does.
Args parse(int argc, char** argv) {
  Args a;
  for (int i = 1; i < argc; ++i) {
    const std::string t = argv[i];
    if (t.compare(0, 2, "--") != 0) continue;
    const std::size_t eq = t.find('=');
    if (eq == std::string::npos)
      a.values[t.substr(2)] = "";
    else
      a.values[t.substr(2, eq - 2)] = t.substr(eq + 1);
  }
  return a;
}

struct UsageError {
  std::string what;
};

int integer(const Args& a, const std::string& key, int fallback, int lo, int hi) {
  const std::string s = a.str(key, "");
  if (s.empty()) return fallback;
  std::size_t used = 0;
  long v = 0;
  try {
    v = std::stol(s, &used);
  } catch (const std::exception&) {
    used = 0;
  }
  if (used != s.size() || v < lo || v > hi)
    throw UsageError{"--" + key + " must be an integer in [" + std::to_string(lo) + ", " + std::to_string(hi) + "]"};
  return static_cast<int>(v);
}

double real(const Args& a, const std::string& key, double fallback) {
  const std::string s = a.str(key, "");
  if (s.empty()) return fallback;
  std::size_t used = 0;
  double v = 0.0;
  try {
    v = std::stod(s, &used);
  } catch (const std::exception&) {
    used = 0;
  }
  if (used != s.size()) throw UsageError{"--" + key + " must be a number"};
  return v;
}

struct Config {
  hsi::SyntheticOptions synthetic;
  bool envi = false;
  hsi::EnviReplayOptions replay;
  hsi::Detector detector = hsi::Detector::Sam;
  std::string library_path;
  bool threshold_given = false;
  double threshold = 0.10;
  double pfa = 1e-4;
  double loading = 1e-6;
  hsi::PipelineOptions pipeline;
  int frames = 300, warmup = 30, repeat = 10;
  bool batch = false, autotune = false, quiet = false, lagged = false;
  std::string csv, dump;
  int print = 0;
};

Config configure(const Args& a) {
  Config c;
  const std::string source = a.str("source", "synthetic");
  if (source == "hot") throw UsageError{"--source=hot is not built in this library; use synthetic or envi"};
  if (source != "synthetic" && source != "envi") throw UsageError{"unknown --source=" + source};
  if (source == "envi") {
    c.envi = true;
    const std::string list = a.str("envi", "");
    std::size_t start = 0;
    while (start <= list.size()) {
      const std::size_t comma = std::min(list.find(',', start), list.size());
      if (comma > start) c.replay.hdr_paths.push_back(list.substr(start, comma - start));
      start = comma + 1;
    }
    if (c.replay.hdr_paths.empty()) throw UsageError{"--source=envi needs --envi=<header>[,<header>...]"};
    c.replay.max_resident = integer(a, "resident", 4, 1, 1 << 16);
  }
  c.synthetic.shape.height = integer(a, "height", 512, 1, 1 << 16);
  c.synthetic.shape.width = integer(a, "width", 512, 1, 1 << 16);
  c.synthetic.shape.bands = integer(a, "bands", 128, 1, 256);
  c.synthetic.num_targets = integer(a, "targets", 3, 1, 16);
  c.synthetic.noise_sigma = static_cast<float>(real(a, "noise", 0.01));
  if (!hsi::parse_detector(a.str("detector", "sam"), &c.detector))
    throw UsageError{"--detector must be sam, cem, rx or ace"};
  c.library_path = a.str("library", "");
  c.threshold_given = a.has("threshold") && !a.str("threshold", "").empty();
  const double fallback = c.detector == hsi::Detector::Sam ? 0.10 : 0.5;
  c.threshold = real(a, "threshold", fallback);
  c.pfa = real(a, "pfa", 1e-4);
  if (!(c.pfa > 0.0 && c.pfa < 1.0)) throw UsageError{"--pfa must lie in (0, 1)"};
  c.loading = real(a, "loading", 1e-6);
  if (!(c.loading >= 0.0)) throw UsageError{"--loading must be >= 0"};
  if (!hsi::parse_sam_variant(a.str("variant", "optimized"), &c.pipeline.variant))
    throw UsageError{"--variant must be baseline, optimized or half"};
  if (!hsi::parse_memory_mode(a.str("memory", "copy"), &c.pipeline.memory))
    throw UsageError{"--memory must be copy or zerocopy"};
  c.pipeline.num_streams = integer(a, "streams", 3, 1, 64);
  c.pipeline.prefill = a.has("prefill") ? 1 : 0;
  c.pipeline.detection.threshold = static_cast<float>(c.threshold);
  c.pipeline.detection.nms_radius = integer(a, "nms", 2, 0, 1 << 15);
  c.pipeline.detection.max_detections = integer(a, "max-detections", 4096, 0, 1 << 30);
  c.pipeline.return_score_map = a.has("dump-score");
  c.frames = integer(a, "frames", 300, 1, 1 << 30);
  c.warmup = integer(a, "warmup", 30, 0, 1 << 30);
  c.batch = a.has("batch");
  c.repeat = integer(a, "repeat", 10, 1, 1 << 20);
  c.autotune = a.has("autotune");
  c.quiet = a.has("quiet");
  c.csv = a.str("csv", a.has("csv") ? "timings.csv" : "");
  c.dump = a.str("dump-score", a.has("dump-score") ? "score.f32" : "");
  c.print = integer(a, "print-detections", 0, 0, 1 << 30);
  c.lagged = a.has("lagged");
  if (c.lagged) {
    if (c.detector == hsi::Detector::Sam) throw UsageError{"--lagged needs --detector=cem, rx or ace"};
    if (c.batch) throw UsageError{"--lagged and --batch are separate modes"};
    if (c.detector == hsi::Detector::Rx && c.threshold_given)
      throw UsageError{"--lagged sets the RX threshold from --pfa; drop --threshold"};
  }
  if (c.batch) {
    if (c.detector == hsi::Detector::Cem)
      throw UsageError{"--batch lists SAM, ACE and RX detections; run --detector=cem without --batch"};
    if (c.frames > 64) throw UsageError{"--batch takes at most 64 frames"};
  }
  return c;
}

void print_device() {
  int device = 0, sms = 0, integrated = 0, mem_khz = 0, bus_bits = 0;
  cudaDeviceProp p{};
  if (cudaGetDevice(&device) != cudaSuccess || cudaGetDeviceProperties(&p, device) != cudaSuccess) {
    std::puts("device: unavailable");
    return;
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&integrated, cudaDevAttrIntegrated, device);
  cudaDeviceGetAttribute(&mem_khz, cudaDevAttrMemoryClockRate, device);
  cudaDeviceGetAttribute(&bus_bits, cudaDevAttrGlobalMemoryBusWidth, device);
  // double data rate: two transfers per memory clock
  const double peak_gbs = 2.0 * mem_khz * (bus_bits / 8.0) / 1.0e6;
  std::printf("device: %s  sm_%d%d  %d SMs  %.1f GB/s peak  %s memory\n", p.name, p.major, p.minor, sms, peak_gbs,
              integrated ? "integrated" : "discrete");
}

// Per-frame timings and the end-of-run report, shared by the three modes.
struct Report {
  std::vector<double> wall_ms;
  double sum_source = 0, sum_upload = 0, sum_score = 0, sum_detect = 0, sum_download = 0, sum_gpu = 0;
  std::uint64_t detections = 0;

  void add(const hsi::FrameResult& r) {
    wall_ms.push_back(r.ms_wall);
    sum_source += r.ms_source;
    sum_upload += r.ms_upload;
    sum_score += r.ms_score;
    sum_detect += r.ms_detect;
    sum_download += r.ms_download;
    sum_gpu += r.ms_gpu;
    detections += r.detections_found;
  }

  void print(const char* score_stage, double wall_s, hsi::CubeShape shape, bool half) const {
    const std::size_t n = wall_ms.size();
    std::vector<double> s = wall_ms;
    std::sort(s.begin(), s.end());
    auto pct = [&](double q) { return n ? s[std::min(n - 1, static_cast<std::size_t>(q * (n - 1) + 0.5))] : 0.0; };
    const double fps = wall_s > 0 ? n / wall_s : 0.0;
    const double cube_gb = static_cast<double>(shape.elements()) * (half ? 2 : 4) * fps / 1e9;
    const double mpix = static_cast<double>(shape.pixels()) * fps / 1e6;
    const double d = n ? static_cast<double>(n) : 1.0;
    std::printf(
        "\nframes %zu in %.3f s\n"
        "  throughput   %.1f fps   %.2f GB/s cube   %.1f Mpixel/s\n"
        "  latency ms   p50 %.3f   p95 %.3f   p99 %.3f   max %.3f\n"
        "  stage ms     source %.3f  upload %.3f  %s %.3f  detect %.3f  download %.3f  gpu %.3f\n"
        "  detections   %llu total, %.1f per frame\n",
        n, wall_s, fps, cube_gb, mpix, pct(0.50), pct(0.95), pct(0.99), n ? s.back() : 0.0, sum_source / d,
        sum_upload / d, score_stage, sum_score / d, sum_detect / d, sum_download / d, sum_gpu / d,
        static_cast<unsigned long long>(detections), n ? static_cast<double>(detections) / d : 0.0);
  }
};

void csv_header(std::ofstream& csv) {
  csv << "frame,detections,ms_source,ms_upload,ms_score,ms_detect,ms_download,ms_gpu,ms_wall\n";
}

void csv_row(std::ofstream& csv, const hsi::FrameResult& r) {
  csv << r.meta.index << "," << r.detections_found << "," << r.ms_source << "," << r.ms_upload << "," << r.ms_score
      << "," << r.ms_detect << "," << r.ms_download << "," << r.ms_gpu << "," << r.ms_wall << "\n";
}

void print_detections(const std::vector<hsi::Detection>& d, int count, const char* unit) {
  std::printf("\nlast frame, first %d of %zu detections:\n", count, d.size());
  for (int i = 0; i < count && i < static_cast<int>(d.size()); ++i)
    std::printf("  (%4d,%4d) target %d  %s %.4f\n", d[i].x, d[i].y, d[i].target, unit, d[i].score);
}

void dump_map(const std::string& path, const std::vector<float>& map, hsi::CubeShape shape) {
  std::ofstream out(path, std::ios::binary);
  out.write(reinterpret_cast<const char*>(map.data()), static_cast<std::streamsize>(map.size() * sizeof(float)));
  std::printf("\nwrote %zu x float32 score map to %s (%dx%d)\n", map.size(), path.c_str(), shape.height, shape.width);
}

const char* unit_of(hsi::Detector d) {
  switch (d) {
    case hsi::Detector::Sam: return "angle";
    case hsi::Detector::Cem: return "cem";
    case hsi::Detector::Rx: return "rx";
    default: return "ace";
  }
}

#define CLI_CUDA(call, what)                                                         \
  do {                                                                               \
    const cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// SAM through hsi::Pipeline: the reference's own flow.
int run_sam_stream(const Config& c, hsi::FrameSource* source, const hsi::SpectralLibrary& library) {
  std::string error;
  auto pipeline = hsi::Pipeline::create(source, library, c.pipeline, &error);
  if (!pipeline) {
    std::fprintf(stderr, "pipeline setup failed: %s\n", error.c_str());
    return 1;
  }
  if (!c.quiet) {
    print_device();
    std::printf("source: %s\n", source->describe().c_str());
    std::printf("run:    %s\n", pipeline->describe().c_str());
  }
  if (c.warmup > 0 && !pipeline->run(static_cast<std::uint64_t>(c.warmup), nullptr, &error)) {
    std::fprintf(stderr, "warm-up failed: %s\n", error.c_str());
    return 1;
  }
  std::vector<hsi::Detection> last;
  std::vector<float> last_map;
  std::ofstream csv;
  if (!c.csv.empty()) {
    csv.open(c.csv);
    csv_header(csv);
  }
  auto on_frame = [&](const hsi::FrameResult& r) {
    last = r.detections;
    if (!r.score_map.empty()) last_map = r.score_map;
    if (csv.is_open()) csv_row(csv, r);
  };
  if (!pipeline->run(static_cast<std::uint64_t>(c.frames), on_frame, &error)) {
    std::fprintf(stderr, "run failed: %s\n", error.c_str());
    return 1;
  }
  const hsi::PipelineStats st = pipeline->stats();
  std::printf(
      "\nframes %llu in %.3f s\n"
      "  throughput   %.1f fps   %.2f GB/s cube   %.1f Mpixel/s\n"
      "  latency ms   p50 %.3f   p95 %.3f   p99 %.3f   max %.3f\n"
      "  stage ms     source %.3f  upload %.3f  sam %.3f  detect %.3f  download %.3f  gpu %.3f\n"
      "  detections   %llu total, %.1f per frame\n",
      static_cast<unsigned long long>(st.frames), st.wall_s, st.fps, st.cube_gb_per_s, st.mpixel_per_s, st.ms_p50,
      st.ms_p95, st.ms_p99, st.ms_max, st.mean_source, st.mean_upload, st.mean_score, st.mean_detect,
      st.mean_download, st.mean_gpu, static_cast<unsigned long long>(st.total_detections),
      st.frames ? static_cast<double>(st.total_detections) / st.frames : 0.0);
  if (!c.dump.empty() && !last_map.empty()) dump_map(c.dump, last_map, source->shape());
  if (c.print > 0) print_detections(last, c.print, "angle");
  return 0;
}

// CEM, RX or ACE, one frame at a time on one stream: upload, the frame's
// statistics (moments + FP64 factorisation), scoring, detection, download.
int run_stat_stream(const Config& c, hsi::FrameSource* source, const hsi::SpectralLibrary& library) {
  const hsi::CubeShape shape = source->shape();
  if (library.bands() != shape.bands) {
    std::fprintf(stderr, "pipeline setup failed: library has %d bands, the source %d\n", library.bands(),
                 shape.bands);
    return 1;
  }
  const std::size_t stride = hsi::bsq_plane_stride(shape), elems = hsi::bsq_device_elements(shape);
  const std::size_t P = shape.pixels();
  const int cap = c.pipeline.detection.max_detections;
  hsi::DetectionParams dp = c.pipeline.detection;
  dp.polarity = hsi::ScorePolarity::HigherIsBetter;
  if (c.detector == hsi::Detector::Rx && !c.threshold_given)
    dp.threshold = static_cast<float>(hsi::rx_threshold_for_false_alarm_rate(shape.bands, c.pfa));
  float* h_cube = nullptr;
  void* d_cube = nullptr;
  float *d_best = nullptr, *d_rx = nullptr;
  std::int32_t* d_which = nullptr;
  hsi::Detection* d_out = nullptr;
  unsigned int* d_count = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t ev[6] = {};
  struct Release {
    std::vector<void*> dev;
    float* host = nullptr;
    cudaStream_t* s;
    cudaEvent_t* ev;
    ~Release() {
      for (void* p : dev) cudaFree(p);
      if (host) cudaFreeHost(host);
      for (int i = 0; i < 6; ++i)
        if (ev[i]) cudaEventDestroy(ev[i]);
      if (*s) cudaStreamDestroy(*s);
    }
  } release{{}, nullptr, &s, ev};
  CLI_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_cube), sizeof(float) * elems), "pinned cube");
  release.host = h_cube;
  auto dev = [&](void** p, std::size_t bytes, const char* what) {
    CLI_CUDA(cudaMalloc(p, bytes), what);
    release.dev.push_back(*p);
  };
  dev(&d_cube, sizeof(float) * elems, "device cube");
  dev(reinterpret_cast<void**>(&d_best), sizeof(float) * P, "score map");
  dev(reinterpret_cast<void**>(&d_rx), sizeof(float) * P, "rx map");
  dev(reinterpret_cast<void**>(&d_which), sizeof(std::int32_t) * P, "target map");
  dev(reinterpret_cast<void**>(&d_out), sizeof(hsi::Detection) * std::max(cap, 1), "detections");
  dev(reinterpret_cast<void**>(&d_count), sizeof(unsigned int), "count");
  CLI_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  for (cudaEvent_t& e : ev) CLI_CUDA(cudaEventCreate(&e), "event");
  if (!c.quiet) {
    print_device();
    std::printf("source: %s\n", source->describe().c_str());
    std::printf("run:    %s per frame on its own statistics (loading %g), threshold %g, nms %d\n",
                hsi::to_string(c.detector), c.loading, static_cast<double>(dp.threshold), dp.nms_radius);
  }
  hsi::DeviceStatistics stats;
  const float* score = c.detector == hsi::Detector::Rx ? d_rx : d_best;
  const std::int32_t* which = c.detector == hsi::Detector::Rx ? nullptr : d_which;
  // --lagged: the runner holds the maps and lists; frame k scores with frame
  // k-1's statistics (frame 0 with its own)
  struct Lagged {
    hsi_lagged* r = nullptr;
    ~Lagged() {
      if (r) hsi_lagged_destroy(r);
    }
  } lagged;
  const int lagged_list = c.detector == hsi::Detector::Cem ? 1 : (c.detector == hsi::Detector::Ace ? 2 : 3);
  if (c.lagged) {
    const std::vector<float> flat = library.flatten();
    hsi_lagged_options o{};
    o.height = shape.height;
    o.width = shape.width;
    o.bands = shape.bands;
    o.dtype = HSI_F32;
    o.targets = flat.data();
    o.num_targets = library.size();
    o.detectors = c.detector == hsi::Detector::Cem ? HSI_LAGGED_SAM_CEM : HSI_LAGGED_RX_ACE;
    o.loading = c.loading;
    o.sam_threshold = 0.10f;
    o.cem_threshold = static_cast<float>(c.threshold);
    o.ace_threshold = static_cast<float>(c.threshold);
    o.rx_false_alarm_rate = c.pfa;
    o.nms_radius = dp.nms_radius;
    o.capacity = cap;
    int st = 0;
    lagged.r = hsi_lagged_create(&o, &st);
    if (!lagged.r) {
      std::fprintf(stderr, "pipeline setup failed: hsi_lagged_create returned %d (%s)\n", st, hsi_status_string(st));
      return 1;
    }
    hsi_lagged_outputs lo{};
    hsi_lagged_outputs_of(lagged.r, &lo);
    if (c.detector == hsi::Detector::Rx) dp.threshold = lo.rx_threshold;
    if (!c.quiet) std::printf("lagged: frame k scored with frame k-1's statistics (frame 0 with its own)\n");
  }
  Report report;
  std::ofstream csv;
  if (!c.csv.empty()) {
    csv.open(c.csv);
    csv_header(csv);
  }
  std::vector<hsi::Detection> last;
  std::vector<float> last_map;
  double timed_s = 0.0;
  for (int f = 0; f < c.warmup + c.frames; ++f) {
    const bool timed = f >= c.warmup;
    const auto t0 = std::chrono::steady_clock::now();
    hsi::FrameResult r;
    if (!source->read_into(h_cube, stride, &r.meta)) break;
    const auto t1 = std::chrono::steady_clock::now();
    CLI_CUDA(cudaEventRecord(ev[0], s), "event");
    CLI_CUDA(cudaMemcpyAsync(d_cube, h_cube, sizeof(float) * elems, cudaMemcpyHostToDevice, s), "upload");
    CLI_CUDA(cudaEventRecord(ev[1], s), "event");
    const hsi::Detection* list = d_out;
    const unsigned int* list_count = d_count;
    const float* map = score;
    if (c.lagged) {
      CLI_CUDA(cudaEventRecord(ev[2], s), "event");
      const int st = hsi_lagged_push(lagged.r, d_cube, reinterpret_cast<hsi_stream_t>(s));
      if (st != HSI_OK) {
        std::fprintf(stderr, "run failed: lagged frame %llu: %s\n", static_cast<unsigned long long>(r.meta.index),
                     hsi_status_string(st));
        return 1;
      }
      hsi_lagged_outputs lo{};
      hsi_lagged_outputs_of(lagged.r, &lo);
      list = reinterpret_cast<const hsi::Detection*>(lo.detections[lagged_list]);
      list_count = lo.counts + lagged_list;
      map = c.detector == hsi::Detector::Rx ? lo.rx : (c.detector == hsi::Detector::Cem ? lo.cem_best : lo.ace_best);
      CLI_CUDA(cudaEventRecord(ev[3], s), "event");
      CLI_CUDA(cudaEventRecord(ev[4], s), "event");
    } else {
      int status = 0;
      const cudaError_t built = stats.build(d_cube, shape, false, library, c.loading, s, &status);
      if (built != cudaSuccess) {
        std::fprintf(stderr, "run failed: statistics of frame %llu: %s (status %d)\n",
                     static_cast<unsigned long long>(r.meta.index), cudaGetErrorString(built), status);
        return 1;
      }
      CLI_CUDA(cudaEventRecord(ev[2], s), "event");
      if (c.detector == hsi::Detector::Cem)
        CLI_CUDA(hsi::launch_cem(d_cube, shape, false, stats, d_best, d_which, nullptr, P, s), "cem");
      else
        CLI_CUDA(hsi::launch_rx_ace(d_cube, shape, false, stats, d_rx, d_best, d_which, nullptr, P, s), "rx/ace");
      CLI_CUDA(cudaEventRecord(ev[3], s), "event");
      CLI_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned int), s), "count");
      CLI_CUDA(hsi::launch_detect(score, which, shape, dp, d_out, d_count, s), "detect");
      CLI_CUDA(cudaEventRecord(ev[4], s), "event");
    }
    unsigned int found = 0;
    CLI_CUDA(cudaMemcpyAsync(&found, list_count, sizeof(found), cudaMemcpyDeviceToHost, s), "download");
    CLI_CUDA(cudaStreamSynchronize(s), "download");
    const std::size_t kept = std::min<std::size_t>(found, static_cast<std::size_t>(cap));
    r.detections.resize(kept);
    if (kept)
      CLI_CUDA(cudaMemcpyAsync(r.detections.data(), list, sizeof(hsi::Detection) * kept, cudaMemcpyDeviceToHost, s),
               "download");
    CLI_CUDA(cudaEventRecord(ev[5], s), "event");
    CLI_CUDA(cudaStreamSynchronize(s), "download");
    const auto t2 = std::chrono::steady_clock::now();
    r.detections_found = found;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    r.ms_upload = ms;
    cudaEventElapsedTime(&ms, ev[1], ev[3]);
    r.ms_score = ms;  // statistics + scoring
    cudaEventElapsedTime(&ms, ev[3], ev[4]);
    r.ms_detect = ms;
    cudaEventElapsedTime(&ms, ev[4], ev[5]);
    r.ms_download = ms;
    cudaEventElapsedTime(&ms, ev[0], ev[5]);
    r.ms_gpu = ms;
    r.ms_source = std::chrono::duration<float, std::milli>(t1 - t0).count();
    r.ms_wall = std::chrono::duration<float, std::milli>(t2 - t0).count();
    if (!timed) continue;
    timed_s += std::chrono::duration<double>(t2 - t0).count();
    report.add(r);
    if (csv.is_open()) csv_row(csv, r);
    last = std::move(r.detections);
    if (!c.dump.empty() && f == c.warmup + c.frames - 1) {
      last_map.resize(P);
      CLI_CUDA(cudaMemcpy(last_map.data(), map, sizeof(float) * P, cudaMemcpyDeviceToHost), "score map");
    }
  }
  report.print(c.lagged ? (c.detector == hsi::Detector::Cem ? "lagged cem" : "lagged rx/ace")
                        : (c.detector == hsi::Detector::Cem ? "stats+cem" : "stats+rx/ace"),
               timed_s, shape, false);
  if (!c.dump.empty() && !last_map.empty()) dump_map(c.dump, last_map, shape);
  if (c.print > 0) print_detections(last, c.print, unit_of(c.detector));
  return 0;
}

// The --frames frames as one batch (include/hsi_batch.h): one eager run,
// then one captured graph replayed --warmup + --repeat times.
int run_batch(const Config& c, hsi::FrameSource* source, const hsi::SpectralLibrary& library) {
  const hsi::CubeShape shape = source->shape();
  if (library.bands() != shape.bands) {
    std::fprintf(stderr, "pipeline setup failed: library has %d bands, the source %d\n", library.bands(),
                 shape.bands);
    return 1;
  }
  if (library.size() < 1 || library.size() > 16) {
    std::fprintf(stderr, "pipeline setup failed: the batch runner takes 1..16 targets, the library has %d\n",
                 library.size());
    return 1;
  }
  const std::size_t stride = hsi::bsq_plane_stride(shape), elems = hsi::bsq_device_elements(shape);
  const std::vector<float> flat = library.flatten();
  std::vector<void*> cubes;
  hsi_batch* batch = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  struct Release {
    std::vector<void*>* cubes;
    hsi_batch** batch;
    cudaStream_t* s;
    cudaEvent_t *e0, *e1;
    ~Release() {
      if (*batch) hsi_batch_destroy(*batch);
      for (void* p : *cubes) cudaFree(p);
      if (*e0) cudaEventDestroy(*e0);
      if (*e1) cudaEventDestroy(*e1);
      if (*s) cudaStreamDestroy(*s);
    }
  } release{&cubes, &batch, &s, &e0, &e1};
  CLI_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  CLI_CUDA(cudaEventCreate(&e0), "event");
  CLI_CUDA(cudaEventCreate(&e1), "event");
  std::vector<float> host(elems);
  std::vector<hsi_batch_frame> frames;
  for (int f = 0; f < c.frames; ++f) {
    hsi::FrameMeta meta;
    if (!source->read_into(host.data(), stride, &meta)) break;
    void* d = nullptr;
    CLI_CUDA(cudaMalloc(&d, sizeof(float) * elems), "device cube");
    cubes.push_back(d);
    CLI_CUDA(cudaMemcpy(d, host.data(), sizeof(float) * elems, cudaMemcpyHostToDevice), "upload");
    hsi_batch_frame fr{};
    fr.cube = d;
    fr.height = shape.height;
    fr.width = shape.width;
    fr.bands = shape.bands;
    fr.dtype = HSI_F32;
    fr.targets = flat.data();
    fr.num_targets = library.size();
    frames.push_back(fr);
  }
  if (frames.empty()) {
    std::fprintf(stderr, "run failed: the source gave no frames\n");
    return 1;
  }
  hsi_batch_options opt{};
  opt.sam_threshold = c.detector == hsi::Detector::Sam ? static_cast<float>(c.threshold) : 0.10f;
  opt.ace_threshold = c.detector == hsi::Detector::Ace ? static_cast<float>(c.threshold) : 0.5f;
  opt.rx_false_alarm_rate = c.pfa;
  opt.loading = c.loading;
  opt.nms_radius = c.pipeline.detection.nms_radius;
  opt.capacity = c.pipeline.detection.max_detections;
  opt.autotune = c.autotune ? 1 : 0;
  int status = 0;
  batch = hsi_batch_create(frames.data(), static_cast<int>(frames.size()), &opt, &status);
  if (!batch) {
    std::fprintf(stderr, "pipeline setup failed: hsi_batch_create returned %d\n", status);
    return 1;
  }
  if (!c.quiet) {
    print_device();
    std::printf("source: %s\n", source->describe().c_str());
    std::printf("run:    batch of %zu frames, %d targets, one CUDA graph per replay%s\n", frames.size(),
                library.size(), c.autotune ? ", autotuned" : "");
  }
  const hsi_stream_t hs = reinterpret_cast<hsi_stream_t>(s);
  int rc = hsi_batch_run(batch, hs);
  if (rc == HSI_OK) rc = hsi_batch_capture(batch, hs);
  for (int i = 0; rc == HSI_OK && i < c.warmup; ++i) rc = hsi_batch_launch(batch, hs);
  if (rc != HSI_OK) {
    std::fprintf(stderr, "run failed: batch status %d\n", rc);
    return 1;
  }
  CLI_CUDA(cudaStreamSynchronize(s), "warm-up");
  const auto t0 = std::chrono::steady_clock::now();
  CLI_CUDA(cudaEventRecord(e0, s), "event");
  for (int i = 0; rc == HSI_OK && i < c.repeat; ++i) rc = hsi_batch_launch(batch, hs);
  CLI_CUDA(cudaEventRecord(e1, s), "event");
  CLI_CUDA(cudaStreamSynchronize(s), "replays");
  const double wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc != HSI_OK) {
    std::fprintf(stderr, "run failed: batch status %d\n", rc);
    return 1;
  }
  float gpu_ms = 0.0f;
  cudaEventElapsedTime(&gpu_ms, e0, e1);
  const int list = c.detector == hsi::Detector::Sam ? 0 : (c.detector == hsi::Detector::Ace ? 1 : 2);
  std::uint64_t total = 0;
  std::vector<hsi::Detection> last;
  std::vector<float> last_map;
  for (std::size_t i = 0; i < frames.size(); ++i) {
    hsi_batch_outputs o{};
    if (hsi_batch_outputs_of(batch, static_cast<int>(i), &o) != HSI_OK) {
      std::fprintf(stderr, "run failed: outputs of frame %zu\n", i);
      return 1;
    }
    std::uint32_t counts[3] = {0, 0, 0};
    CLI_CUDA(cudaMemcpy(counts, o.counts, sizeof(counts), cudaMemcpyDeviceToHost), "counts");
    total += counts[list];
    if (i + 1 == frames.size()) {
      const std::size_t kept = std::min<std::size_t>(counts[list], static_cast<std::size_t>(opt.capacity));
      last.resize(kept);
      if (kept)
        CLI_CUDA(cudaMemcpy(last.data(), o.detections[list], sizeof(hsi::Detection) * kept, cudaMemcpyDeviceToHost),
                 "detections");
      if (!c.dump.empty()) {
        const float* map = list == 0 ? o.sam_best : (list == 1 ? o.ace_best : o.rx);
        last_map.resize(shape.pixels());
        CLI_CUDA(cudaMemcpy(last_map.data(), map, sizeof(float) * shape.pixels(), cudaMemcpyDeviceToHost),
                 "score map");
      }
    }
  }
  const double per_batch_ms = gpu_ms / c.repeat;
  const double mpix = static_cast<double>(shape.pixels()) * frames.size() / (per_batch_ms * 1e3);
  std::printf(
      "\nbatch of %zu frames, %d replays in %.3f s\n"
      "  throughput   %.2f ms per batch (device)   %.1f Mpixel/s\n"
      "  detections   %llu %s in the batch, %.1f per frame\n",
      frames.size(), c.repeat, wall_s, per_batch_ms, mpix, static_cast<unsigned long long>(total),
      hsi::to_string(c.detector), static_cast<double>(total) / frames.size());
  if (!c.dump.empty() && !last_map.empty()) dump_map(c.dump, last_map, shape);
  if (c.print > 0) print_detections(last, c.print, unit_of(c.detector));
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  const Args args = parse(argc, argv);
  if (args.has("help") || args.has("h")) {
    std::puts(kUsage);
    return 0;
  }
  Config c;
  try {
    c = configure(args);
  } catch (const UsageError& e) {
    std::fprintf(stderr, "%s\n", e.what.c_str());
    return 2;
  }
  try {
    hsi::SpectralLibrary library;
    std::unique_ptr<hsi::FrameSource> source;
    if (!c.library_path.empty()) library = hsi::read_spectra_csv(c.library_path);
    source = c.envi ? hsi::make_envi_replay_source(c.replay) : hsi::make_synthetic_source(c.synthetic);
    if (!source) {
      std::fprintf(stderr, "pipeline setup failed: frame source\n");
      return 1;
    }
    if (c.library_path.empty()) {
      // the synthetic source knows what it planted, so the tool runs with no
      // arguments at all; an ENVI replay needs --library
      if (!source->library()) {
        std::fputs("no target spectra: pass --library=<csv>\n", stderr);
        return 2;
      }
      library = *source->library();
    }
    if (c.batch) return run_batch(c, source.get(), library);
    if (c.detector == hsi::Detector::Sam) return run_sam_stream(c, source.get(), library);
    return run_stat_stream(c, source.get(), library);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
