// nbody_cli.cpp -- command-line driver with the reference's interface
// (apps/simulation/main.cpp:44-333 of sytrams/AMSC-Nbody): same options,
// output lines and exit codes (0 success, 2 argument error with usage, 1
// runtime failure).  --stream-dir, --sample-rate and --stream-max-particles
// write quantized frames to a spool directory as the reference does; its
// stream server options (--cluster, --stream-bind, --stream-port,
// --stream-server) belong to a viewer stack this library does not provide
// and are rejected as argument errors.  Additions: --precision and
// --gravitational-constant.
#include <cerrno>
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <string_view>

#include "nbb_simulation.hpp"
#include "nbb_streaming.hpp"

namespace {

struct Options {
  std::string inputPath;
  std::size_t steps = 0;
  SimulationConfig simulation{0.0, 0.5, 1.0e-6};
  SimulationOptions extra{};
  std::string streamDirectory;
  double sampleRate = 60.0;
  std::size_t maximumStreamParticles = 100000;
  bool streamEnabled = false;
  bool showHelp = false;
  bool hasTimeStep = false;
  bool hasSteps = false;
};

void printUsage(std::ostream &out, const char *program) {
  out << "Usage:\n"
      << "  " << program << " --input FILE --time-step DT --steps N [OPTIONS]\n\n"
      << "Required arguments:\n"
      << "  -i, --input FILE       Binary particle input file\n"
      << "  -t, --time-step DT     Positive shared simulation timestep\n"
      << "  -n, --steps N          Positive number of timesteps\n\n"
      << "Force options:\n"
      << "      --theta VALUE      Barnes-Hut opening angle (default: 0.5)\n"
      << "      --softening VALUE  Non-negative softening length (default: 1e-6)\n"
      << "      --precision MODE   fp64 (reference arithmetic) or mixed (default: fp64)\n"
      << "      --gravitational-constant VALUE  G (default: 6.6743e-11)\n\n"
      << "Frame output options:\n"
      << "      --stream-dir DIR   Durable frame queue; also enables output\n"
      << "      --sample-rate HZ   Maximum wall-clock sample rate (default: 60)\n"
      << "      --stream-max-particles N  Frame sample size; 0 writes all (default: 100000)\n\n"
      << "Other options:\n"
      << "  -h, --help             Show this help and exit\n";
}

std::string_view requireValue(int argc, char **argv, int &index, std::string_view option) {
  if (index + 1 >= argc) throw std::invalid_argument("Missing value for " + std::string(option));
  return argv[++index];
}

double parseDouble(std::string_view text, std::string_view option) {
  const std::string s(text);
  char *end = nullptr;
  errno = 0;
  const double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str() || *end != '\0' || errno == ERANGE || !std::isfinite(v))
    throw std::invalid_argument("Invalid numeric value for " + std::string(option) + ": " + s);
  return v;
}

std::size_t parseNonNegativeCount(std::string_view text, std::string_view option) {
  std::size_t v = 0;
  const auto r = std::from_chars(text.data(), text.data() + text.size(), v);
  if (r.ec != std::errc{} || r.ptr != text.data() + text.size())
    throw std::invalid_argument("Invalid non-negative integer for " + std::string(option) + ": " + std::string(text));
  return v;
}

std::size_t parseStepCount(std::string_view text, std::string_view option) {
  std::size_t v = 0;
  const auto r = std::from_chars(text.data(), text.data() + text.size(), v);
  if (r.ec != std::errc{} || r.ptr != text.data() + text.size() || v == 0)
    throw std::invalid_argument("Invalid positive integer for " + std::string(option) + ": " + std::string(text));
  return v;
}

Options parseCommandLine(int argc, char **argv) {
  Options o;
  for (int i = 1; i < argc; ++i) {
    const std::string_view opt(argv[i]);
    if (opt == "-h" || opt == "--help") {
      o.showHelp = true;
      return o;
    }
    if (opt == "-i" || opt == "--input") {
      o.inputPath = requireValue(argc, argv, i, opt);
    } else if (opt == "-t" || opt == "--time-step") {
      o.simulation.timeStep = parseDouble(requireValue(argc, argv, i, opt), opt);
      o.hasTimeStep = true;
    } else if (opt == "-n" || opt == "--steps") {
      o.steps = parseStepCount(requireValue(argc, argv, i, opt), opt);
      o.hasSteps = true;
    } else if (opt == "--theta") {
      o.simulation.theta = parseDouble(requireValue(argc, argv, i, opt), opt);
    } else if (opt == "--softening") {
      o.simulation.softening = parseDouble(requireValue(argc, argv, i, opt), opt);
    } else if (opt == "--gravitational-constant") {
      o.extra.gravitationalConstant = parseDouble(requireValue(argc, argv, i, opt), opt);
    } else if (opt == "--precision") {
      const std::string_view v = requireValue(argc, argv, i, opt);
      if (v == "fp64") {
        o.extra.precision = NBB_PRECISION_FP64;
      } else if (v == "mixed") {
        o.extra.precision = NBB_PRECISION_MIXED;
      } else {
        throw std::invalid_argument("Invalid value for --precision: " + std::string(v));
      }
    } else if (opt == "--stream-dir") {
      o.streamDirectory = requireValue(argc, argv, i, opt);
      o.streamEnabled = true;
    } else if (opt == "--sample-rate") {
      o.sampleRate = parseDouble(requireValue(argc, argv, i, opt), opt);
    } else if (opt == "--stream-max-particles") {
      o.maximumStreamParticles = parseNonNegativeCount(requireValue(argc, argv, i, opt), opt);
    } else if (opt == "--cluster" || opt == "--stream-bind" || opt == "--stream-port" || opt == "--stream-server") {
      throw std::invalid_argument("The stream server is not part of this build: " + std::string(opt));
    } else {
      throw std::invalid_argument("Unknown option: " + std::string(opt));
    }
  }
  if (o.inputPath.empty()) throw std::invalid_argument("--input is required");
  if (!o.hasTimeStep) throw std::invalid_argument("--time-step is required");
  if (!o.hasSteps) throw std::invalid_argument("--steps is required");
  if (o.simulation.timeStep <= 0.0) throw std::invalid_argument("--time-step must be positive");
  if (o.simulation.theta < 0.0) throw std::invalid_argument("--theta must be non-negative");
  if (o.simulation.softening < 0.0) throw std::invalid_argument("--softening must be non-negative");
  if (o.sampleRate <= 0.0) throw std::invalid_argument("--sample-rate must be positive");
  if (o.streamEnabled && o.streamDirectory.empty()) throw std::invalid_argument("--stream-dir must not be empty");
  return o;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    const Options options = parseCommandLine(argc, argv);
    if (options.showHelp) {
      printUsage(std::cout, argv[0]);
      return 0;
    }
    std::ifstream input(options.inputPath, std::ios::binary);
    if (!input.is_open()) throw std::runtime_error("Could not open particle input file: " + options.inputPath);
    std::unique_ptr<nbody::streaming::FrameSpool> spool;
    std::unique_ptr<nbody::streaming::FrameSampler> sampler;
    if (options.streamEnabled) {
      spool = std::make_unique<nbody::streaming::FrameSpool>(options.streamDirectory);
      sampler = std::make_unique<nbody::streaming::FrameSampler>(options.sampleRate);
    }
    Particles particles(input);
    const std::size_t count = particles.size();
    Simulation simulation(std::move(particles), options.simulation, options.extra);
    std::unique_ptr<nbody::streaming::DeviceFrameWriter> writer;
    if (spool) writer = std::make_unique<nbody::streaming::DeviceFrameWriter>(simulation, options.maximumStreamParticles);
    std::cout << "Loaded " << count << " particles from " << options.inputPath << '\n';
    const auto initStart = std::chrono::steady_clock::now();
    simulation.initialize();
    const auto initEnd = std::chrono::steady_clock::now();
    std::size_t framesWritten = 0;
    std::size_t lastCaptured = std::numeric_limits<std::size_t>::max();
    auto capture = [&](bool force) {
      if (!sampler) return;
      const std::chrono::duration<double> elapsed = std::chrono::steady_clock::now() - initEnd;
      if (!force && !sampler->isDue(elapsed.count())) return;
      (void)writer->write(*spool, sampler->takeSequence());
      ++framesWritten;
      lastCaptured = simulation.stepNumber();
    };
    capture(false);
    for (std::size_t s = 0; s < options.steps; ++s) {
      simulation.step();
      capture(false);
    }
    if (sampler && lastCaptured != simulation.stepNumber()) capture(true);
    if (spool) (void)spool->markComplete();
    const auto evolEnd = std::chrono::steady_clock::now();
    const std::chrono::duration<double> initElapsed = initEnd - initStart;
    const std::chrono::duration<double> evolElapsed = evolEnd - initEnd;
    const std::chrono::duration<double> total = evolEnd - initStart;
    std::cout << std::setprecision(17) << "Simulation complete\n"
              << "  steps: " << simulation.stepNumber() << '\n'
              << "  simulated time: " << simulation.time() << '\n'
              << "  initialization wall time: " << initElapsed.count() << " seconds\n"
              << "  evolution wall time: " << evolElapsed.count() << " seconds\n"
              << "  average step time: " << 1000.0 * evolElapsed.count() / static_cast<double>(options.steps)
              << " ms\n"
              << "  total wall time: " << total.count() << " seconds\n";
    if (spool) {
      std::cout << "  frames written: " << framesWritten << '\n'
                << "  particles per frame: " << writer->sampleParticleCount() << " of " << count << '\n'
                << "  frame spool: " << spool->directory() << '\n';
    }
    return 0;
  } catch (const std::invalid_argument &error) {
    std::cerr << "Argument error: " << error.what() << "\n\n";
    printUsage(std::cerr, argv[0]);
    return 2;
  } catch (const std::exception &error) {
    std::cerr << "Simulation failed: " << error.what() << '\n';
    return 1;
  }
}
