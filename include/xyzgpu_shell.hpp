// The reference renderer's command shell and .ren scripts (xyz/core/shell.cpp:
// 204-497, xyz/main.cpp:54-63) over the xyzgpu C ABI: the same commands with
// the same meaning, so a user's .ren scripts drive the GPU path tracer.
// Header-only host C++; link with libxyzgpu.so.  The program
// xyz_b200/xyzgpu_shell (xyz_b200/csrc/shell_main.cpp) wraps it like the
// reference's xyz.exe.
//
// Commands (one per line; blank lines, lines starting with "rem " and
// blocks from "=begin" to "=end" are skipped):
//   load NAME         Scene::Load of <mqo dir>/NAME.mqo and Scene::Build (the
//                     kd-tree); the document's Scene chunk sets the camera.
//                     Extension: NAME.ply when there is no NAME.mqo (the
//                     reference converts PLY with its ply2mqo tool first).
//   save NAME         writes <ren dir>/NAME.ren: the script that repeats this
//                     state (load, eye, at, dim, it, rt, rep, ren)
//   set eye X Y Z     ThinLensCamera::MoveTo
//   set at X Y Z      ThinLensCamera::LookAt
//   set dim W H       Scene::SetDimension (values below 1 become 1)
//   set rt TIME       rendering time; raises `it` to it when shorter
//   set it TIME       interval between saved images; raises `rt` likewise
//                     (TIME: "<n> <unit>" pairs, units d/day/days, h/hr/hour/
//                     hours, m/min/minute/minutes, s/sec/second/seconds)
//   set rep N         algorithm: 0 path tracing (PathTracer), 1 importance-
//                     driven path tracing (ImportanceDrivenPathTracer); the
//                     reference's 2-14 (MLT, bidirectional and population
//                     variants) are not built and are refused with a message
//   ren               renders for `rt` seconds when rt > 0 into the folder
//                     <out dir>/<program>/<scene> WWWWxHHHH YYYY-MM-DDThh.mm.ss
//                     PT/ (IDPT/ for rep 1), saving the film as
//                     "hhHmmMssS SSSSSSspp NNNNNNNNNNNN.pfm" (time, samples per
//                     pixel, rays traced) after every `it` seconds and at the end
//   quit              ends an interactive shell; no effect in a script (as in
//                     the reference, whose scripts continue after it)
//   exit              ends the shell
//   abort             as quit
//   Extensions with no counterpart in the reference (its random numbers come
//   from one global std::mt19937_64 and its run is bounded by time only):
//   set spp N         also stop once N samples per pixel are done (0: no bound)
//   set seed S        seed of the render's Philox streams and of the importon
//                     particles
// Differences: time is wall-clock seconds on the host (the reference counts
// process CPU time with std::clock, which includes its own rendering); a pass
// over the image renders several samples per pixel on the GPU (the reference
// checks the time after every single sample per pixel), chosen so a pass takes
// a fraction of the interval; the film holds the same sums whatever the pass
// sizes.  Failures print a message and the shell continues, as the reference's
// do.
#pragma once

#include <sys/stat.h>

#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <ctime>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>

#include "xyzgpu.h"
#include "xyzgpu_mqo.hpp"
#include "xyzgpu_scene.hpp"

namespace xyzgpu {

namespace shell_detail {

// stream2time (shell.cpp:19-47): sums "<value> <unit>" pairs into seconds;
// a pair with an unknown unit adds nothing.
inline int StreamToTime(std::istream &in) {
  int time = 0;
  while (in) {
    int val;
    in >> val;
    if (!in) break;
    std::string unit;
    in >> unit;
    if (unit == "d" || unit == "day" || unit == "days")
      time += val * (60 * 60 * 24);
    else if (unit == "h" || unit == "hr" || unit == "hour" || unit == "hours")
      time += val * (60 * 60);
    else if (unit == "m" || unit == "min" || unit == "minute" || unit == "minutes")
      time += val * 60;
    else if (unit == "s" || unit == "sec" || unit == "second" || unit == "seconds")
      time += val;
  }
  return time;
}

// time2string (shell.cpp:49-84): "1 day 2 hours 3 minutes 4 seconds" with the
// zero parts left out; zero itself is " 0 s".
inline std::string TimeToString(int time) {
  int const days = time / (60 * 60 * 24);
  int const hours = (time / (60 * 60)) % 24;
  int const minutes = (time / 60) % 60;
  int const seconds = time % 60;
  std::ostringstream out;
  if (days > 0) out << days << (days > 1 ? " days" : " day");
  if (hours > 0) out << (days > 0 ? " " : "") << hours << (hours > 1 ? " hours" : " hour");
  if (minutes > 0) out << (days > 0 || hours > 0 ? " " : "") << minutes << (minutes > 1 ? " minutes" : " minute");
  if (seconds > 0)
    out << (days > 0 || hours > 0 || minutes > 0 ? " " : "") << seconds << (seconds > 1 ? " seconds" : " second");
  if (days == 0 && hours == 0 && minutes == 0 && seconds == 0) out << " 0 s";
  return out.str();
}

// hi::mkdir (libhi/hi/file/file.cpp:5-27): makes every folder on the path;
// false when one cannot be made and does not exist.
inline bool MakeDirs(std::string dir) {
  auto make = [&]() { return ::mkdir(dir.c_str(), 0777) == 0 || errno == EEXIST; };
  for (size_t i = 0; i < dir.size(); ++i) {
    if (dir[i] == '/' || dir[i] == '\\') {
      char const c = dir[i];
      dir[i] = '\0';
      bool const ok = dir.c_str()[0] == '\0' || make();
      dir[i] = c;
      if (!ok) return false;
    }
  }
  return make();
}

// hi::path2name (file.cpp:71-91): the file name without folder and extension.
inline std::string PathToName(std::string path) {
  for (char &c : path)
    if (c == '\\') c = '/';
  size_t const dot = path.find_last_of('.');
  if (dot != std::string::npos) path.resize(dot);
  size_t const slash = path.find_last_of('/');
  if (slash != std::string::npos) path.erase(0, slash + 1);
  return path;
}

inline bool StartsWith(const std::string &s, const char *p) { return s.compare(0, std::strlen(p), p) == 0; }

}  // namespace shell_detail

class Shell {
 public:
  enum Result { kExit, kQuit, kContinue, kUnknown };

  struct Config {
    std::string mqo_dir = "./";            // MQODIR_PATH (xyz/core/config.hpp:17)
    std::string ren_dir = "./";            // RENDIR_PATH
    std::string out_dir = "./";            // OUTDIR_PATH
    std::string program = "xyzgpu_shell";  // the folder named for the program
    std::ostream *log = &std::cerr;
  };

  Shell() : Shell(Config()) {}
  explicit Shell(Config cfg) : cfg_(std::move(cfg)) { ReferenceLightPowerXYZ(power_); }
  ~Shell() { Unload(); }
  Shell(const Shell &) = delete;
  Shell &operator=(const Shell &) = delete;

  // Shell(in, gui) (shell.cpp:451-497) reading a script (interactive =
  // false: quit has no effect) or a terminal (interactive = true: quit
  // returns).  Returns 0 at the end of the input and at exit.
  int Run(std::istream &in, bool interactive = false) {
    std::string line;
    for (;;) {
      *cfg_.log << "\n[XYZGPU]> " << std::flush;
      do {
        if (!std::getline(in, line)) {
          *cfg_.log << "Bye Bye" << std::endl;
          return 0;
        }
        mqo_detail::trim(line);
        if (line == "=begin") {
          do {
            if (!std::getline(in, line)) {
              *cfg_.log << "bye-bye" << std::endl;
              return 0;
            }
            mqo_detail::trim(line);
          } while (line != "=end");
          line.clear();
        }
      } while (line.empty() || shell_detail::StartsWith(line, "rem "));
      switch (Interpret(line)) {
        case kExit:
          return 0;
        case kQuit:
          if (interactive) return 0;
          break;
        case kContinue:
          break;
        default:
          *cfg_.log << "undefined" << std::endl;
          break;
      }
      *cfg_.log << std::endl;
    }
  }

  // Interpret (shell.cpp:204-448): one command line.
  Result Interpret(const std::string &command_line) {
    std::istringstream sin(command_line);
    std::string command;
    sin >> command;
    if (command == "quit") return kQuit;
    if (command == "exit") return kExit;
    if (command == "abort") return kQuit;
    try {
      if (command == "set") return Set(sin);
      if (command == "load") {
        sin >> scene_name_;
        Load();
        return kContinue;
      }
      if (command == "save") {
        std::string name;
        sin >> name;
        Save(name);
        return kContinue;
      }
      if (command == "ren") return Ren();
    } catch (const Error &e) {
      *cfg_.log << "error: " << e.what() << std::endl;
      return kContinue;
    }
    return kUnknown;
  }

  // State, for programs that drive the shell.
  const std::string &SceneName() const { return scene_name_; }
  const std::string &OutdirPath() const { return outdir_path_; }
  const std::string &LastImage() const { return last_image_; }
  int RenderingTime() const { return rendering_time_; }
  int IntervalTime() const { return interval_time_; }
  int Algorithm() const { return algorithm_; }
  int Width() const { return width_; }
  int Height() const { return height_; }
  const xyzgpu_camera &Camera() const { return camera_.desc(); }
  int SamplesDone() const { return spp_done_; }
  bool Loaded() const { return scene_ != nullptr; }

 private:
  Result Set(std::istringstream &sin) {
    std::string what;
    sin >> what;
    std::ostream &log = *cfg_.log;
    if (what == "rep") {
      sin >> algorithm_;
      log << "rep (" << algorithm_ << ")";
    } else if (what == "rt") {
      rendering_time_ = shell_detail::StreamToTime(sin);
      if (interval_time_ > rendering_time_) interval_time_ = rendering_time_;
      log << "it (" << interval_time_ << "), rt (" << rendering_time_ << ")";
    } else if (what == "it") {
      interval_time_ = shell_detail::StreamToTime(sin);
      if (interval_time_ > rendering_time_) rendering_time_ = interval_time_;
      log << "it (" << interval_time_ << "), rt (" << rendering_time_ << ")";
    } else if (what == "eye") {
      float e[3] = {0, 0, 0};
      sin >> e[0] >> e[1] >> e[2];
      camera_.MoveTo(e[0], e[1], e[2]);
      log << "eye (" << e[0] << ", " << e[1] << ", " << e[2] << ")";
    } else if (what == "at") {
      float a[3] = {0, 0, 0};
      sin >> a[0] >> a[1] >> a[2];
      camera_.LookAt(a[0], a[1], a[2]);
      log << "at (" << a[0] << ", " << a[1] << ", " << a[2] << ")";
    } else if (what == "dim") {
      int w = 0, h = 0;
      sin >> w >> h;
      width_ = w <= 0 ? 1 : w;
      height_ = h <= 0 ? 1 : h;
      log << "dim (" << width_ << ", " << height_ << ")";
    } else if (what == "spp") {
      sin >> spp_limit_;
      if (spp_limit_ < 0) spp_limit_ = 0;
      log << "spp (" << spp_limit_ << ")";
    } else if (what == "seed") {
      sin >> seed_;
      log << "seed (" << seed_ << ")";
    }
    return kContinue;
  }

  void Unload() {
    if (scene_) xyzgpu_scene_destroy(scene_);
    scene_ = nullptr;
  }

  static double Seconds(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
  }

  // load (shell.cpp:273-313): parse, then build the kd-tree on the GPU.
  void Load() {
    std::string path = cfg_.mqo_dir + scene_name_ + ".mqo";
    bool ply = false;
    std::ifstream in(path, std::ios::binary);
    if (!in) {
      path = cfg_.mqo_dir + scene_name_ + ".ply";
      in.open(path, std::ios::binary);
      ply = true;
    }
    if (!in) return;  // the reference ignores a scene it cannot open
    std::ostream &log = *cfg_.log;
    log << "\nload scene (" << path << ") ... " << std::endl;
    auto const t0 = std::chrono::steady_clock::now();
    MqoScene sc;
    std::string err;
    if (!(ply ? LoadPly(in, &sc, &err) : LoadMqo(in, &sc, &err))) throw Error(XYZGPU_E_INVALID, path + ": " + err);
    auto const t1 = std::chrono::steady_clock::now();
    log << "done: " << Seconds(t0, t1) << " s, " << sc.tri_material.size() << " triangles\n";
    log << "build kd-tree ... ";
    Unload();
    xyzgpu_build_params bp;
    xyzgpu_build_params_default(&bp);
    xyzgpu_scene_desc const d = sc.Desc(power_);
    check(xyzgpu_scene_create(&d, &bp, &scene_));
    auto const t2 = std::chrono::steady_clock::now();
    log << "done: " << Seconds(t1, t2) << " s";
    if (sc.has_camera) {
      camera_.MoveTo(sc.eye[0], sc.eye[1], sc.eye[2]);
      camera_.LookAt(sc.at[0], sc.at[1], sc.at[2]);
    }
    specular_ = false;
    for (auto const &m : sc.materials) specular_ = specular_ || (!m.light && m.kind != XYZGPU_MATERIAL_LAMBERT);
  }

  // save (shell.cpp:315-346).
  void Save(const std::string &name) {
    shell_detail::MakeDirs(cfg_.ren_dir);
    std::ofstream fout(cfg_.ren_dir + name + ".ren");
    if (!fout) return;
    const xyzgpu_camera &c = camera_.desc();
    fout << "load " << scene_name_ << "\n\n";
    fout << "set eye " << c.eye[0] << ' ' << c.eye[1] << ' ' << c.eye[2] << "\n";
    fout << "set at  " << c.at[0] << ' ' << c.at[1] << ' ' << c.at[2] << "\n\n";
    fout << "set dim " << width_ << ' ' << height_ << "\n";
    fout << "set it  " << shell_detail::TimeToString(interval_time_) << "\n";
    fout << "set rt  " << shell_detail::TimeToString(rendering_time_) << "\n\n";
    fout << "set rep " << algorithm_ << "\n";
    fout << "ren\n";
  }

  // ren (shell.cpp:348-447) with the integrators' loop (PathTracer::run,
  // ImportanceDrivenPathTracer::run, xyz/integrator/integrator.cpp:88-253).
  Result Ren() {
    if (rendering_time_ <= 0) return kContinue;
    static const char *const kFolders[] = {"PT/",    "IDPT/",    "PT_MLT/",    "IDPT_MLT/", "PTwGW/",
                                           "IDPTwGW/", "PTwGW_MLT/", "IDPTwGW_MLT/", "BPT/",      "IDBPT/",
                                           "BPT_MLT/", "IDBPT_MLT/", "MLT/",        "PT_PLT/",   "BPT_PLT/"};
    if (algorithm_ < 0 || algorithm_ > 14) return kContinue;
    if (algorithm_ > 1) {
      *cfg_.log << "rep " << algorithm_ << " (" << kFolders[algorithm_]
                << ") is not available: the GPU tracer has path tracing (0) and importance-driven path tracing (1)"
                << std::endl;
      return kContinue;
    }
    if (!scene_) throw Error(XYZGPU_E_INVALID, "ren: no scene is loaded");
    {
      std::time_t now = std::time(nullptr);
      std::tm t;
      localtime_r(&now, &t);
      char buf[1024];
      std::snprintf(buf, sizeof(buf), "%s%s/%s %04dx%04d %04d-%02d-%02dT%02d.%02d.%02d ", cfg_.out_dir.c_str(),
                    cfg_.program.c_str(), scene_name_.c_str(), width_, height_, 1900 + t.tm_year, 1 + t.tm_mon,
                    t.tm_mday, t.tm_hour, t.tm_min, t.tm_sec);
      outdir_path_ = std::string(buf) + kFolders[algorithm_];
    }
    *cfg_.log << "mkdir: `" << outdir_path_ << "'" << std::endl;
    if (!shell_detail::MakeDirs(outdir_path_)) {
      *cfg_.log << "cannot make the output folder (" << outdir_path_ << ")" << std::endl;
      return kContinue;
    }
    Render(algorithm_ == 1);
    return kQuit;
  }

  void Render(bool importance) {
    std::ostream &log = *cfg_.log;
    xyzgpu_importons map = nullptr;
    struct MapGuard {
      xyzgpu_importons *m;
      ~MapGuard() {
        if (*m) xyzgpu_importons_destroy(*m);
      }
    } guard{&map};
    if (importance) {
      log << "** Importance Driven Path Tracing **\n>>>> Build Importance Map <<<<\n";
      if (specular_) throw Error(XYZGPU_E_INVALID, "rep 1: the importon tracer takes Lambert scenes only");
      xyzgpu_importon_config cfg;
      xyzgpu_importon_config_default(&cfg);
      cfg.seed = seed_;
      check(xyzgpu_importons_create(scene_, &cfg, nullptr, 0, nullptr, &map));
    } else {
      log << "** Path Tracing **\n";
    }
    log << ">>>> Computation <<<<\n";
    ImageFilm film(width_, height_);
    xyzgpu_render_params rp;
    xyzgpu_render_params_default(&rp);
    rp.width = width_;
    rp.height = height_;
    rp.seed = seed_;
    rp.film_location = XYZGPU_FILM_HOST;
    rp.accumulate = 1;
    // a pass targets a quarter of the interval, at most half a second
    double const target = interval_time_ > 0 ? std::min(0.5, interval_time_ / 4.0) : 0.5;
    int chunk = 1;
    unsigned long long rays = 0;
    int save_time = interval_time_;
    spp_done_ = 0;
    auto begin = std::chrono::steady_clock::now();
    for (;;) {
      rp.spp = spp_limit_ > 0 ? std::min(chunk, spp_limit_ - spp_done_) : chunk;
      rp.spp_offset = spp_done_;
      auto const p0 = std::chrono::steady_clock::now();
      if (map)
        check(xyzgpu_render_importon(map, &camera_.desc(), &rp, film.data(), nullptr));
      else
        check(xyzgpu_render(scene_, &camera_.desc(), &rp, film.data(), nullptr));
      xyzgpu_render_counters rc;
      check(xyzgpu_render_counters_get(scene_, &rc));
      rays += rc.extension_rays + rc.shadow_rays;
      spp_done_ += rp.spp;
      auto const p1 = std::chrono::steady_clock::now();
      double const pass = Seconds(p0, p1);
      if (pass < target / 2 && chunk < 1024) chunk *= 2;
      if (pass > target * 2 && chunk > 1) chunk /= 2;
      double const elapsed = Seconds(begin, p1);
      int const time = static_cast<int>(elapsed + 0.5);
      char line[128];
      std::snprintf(line, sizeof(line), "\r  %02dh%02dm%02ds %+6d[spp]", time / 3600, (time / 60) % 60, time % 60,
                    spp_done_);
      log << line << std::flush;
      bool const finished = spp_limit_ > 0 && spp_done_ >= spp_limit_;
      if (finished || time >= save_time) {
        save_time += interval_time_;
        char name[128];
        std::snprintf(name, sizeof(name), "%02dh%02dm%02ds %06dspp %012llu.pfm", time / 3600, (time / 60) % 60,
                      time % 60, spp_done_, rays);
        last_image_ = outdir_path_ + name;
        if (!film.Save(last_image_, static_cast<float>(spp_done_)))
          throw Error(XYZGPU_E_INVALID, "cannot write " + last_image_);
        if (finished || time >= rendering_time_) break;
        // the time spent saving is not rendering time (integrator.cpp:155)
        begin = std::chrono::steady_clock::now() -
                std::chrono::duration_cast<std::chrono::steady_clock::duration>(std::chrono::duration<double>(elapsed));
      }
    }
    log << std::endl;
  }

  Config cfg_;
  std::string scene_name_, outdir_path_, last_image_;
  int rendering_time_ = 0, interval_time_ = 0, algorithm_ = 0;
  int width_ = 720, height_ = 480;  // Scene::Scene's SetDimension(720, 480)
  int spp_limit_ = 0, spp_done_ = 0;
  uint64_t seed_ = 0;
  float power_[3] = {0, 0, 0};
  bool specular_ = false;
  xyzgpu_scene scene_ = nullptr;
  ThinLensCamera camera_;
};

}  // namespace xyzgpu
