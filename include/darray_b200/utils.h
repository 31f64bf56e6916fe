// The utilities of include/utils.h that DArray's tests use, with the same interfaces: ArgsParser (add_option on an
// int/float/double/string/bool variable with a help string, a long name, a short name and a value name; parse of
// "--long value", "--long=value", "-s value"; --help prints the options), ElapsedTimer (start, elapsed in
// milliseconds) and Tracer (scoped timing events: trace_on/trace_off, a standalone tracer prints its duration,
// save_events_to_file writes "time START|END \"op\"" lines).  Backtraces (the rest of utils.h) are not provided.
#pragma once
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <type_traits>
#include <string>
#include <vector>

namespace DArray {

class ArgsParser {
 public:
  template <typename T>
  void add_option(T& value, const char* help, const char* long_name, char short_name, const char* value_name = nullptr) {
    Option o;
    o.help = help ? help : "";
    o.long_name = long_name ? long_name : "";
    o.short_name = short_name;
    o.value_name = value_name ? value_name : "";
    o.flag = std::is_same<T, bool>::value;
    o.accept = [&value](const char* s) { return assign(value, s); };
    m_options.push_back(o);
  }
  // Returns false (after a message) on an unknown option or a bad value; exits after --help.
  bool parse(int argc, char** argv) {
    for (int i = 1; i < argc; ++i) {
      const char* a = argv[i];
      const Option* o = nullptr;
      const char* val = nullptr;
      if (a[0] == '-' && a[1] == '-') {
        if (!std::strcmp(a + 2, "help")) {
          usage(argv[0]);
          std::exit(0);
        }
        const char* eq = std::strchr(a + 2, '=');
        const std::string name = eq ? std::string(a + 2, eq) : std::string(a + 2);
        for (const Option& x : m_options)
          if (x.long_name == name) o = &x;
        if (eq) val = eq + 1;
      } else if (a[0] == '-' && a[1] && !a[2]) {
        for (const Option& x : m_options)
          if (x.short_name == a[1]) o = &x;
      }
      if (!o) {
        std::fprintf(stderr, "unknown option %s\n", a);
        return false;
      }
      if (o->flag && !val) val = "1";
      if (!val) {
        if (i + 1 >= argc) {
          std::fprintf(stderr, "option %s needs a value\n", a);
          return false;
        }
        val = argv[++i];
      }
      if (!o->accept(val)) {
        std::fprintf(stderr, "bad value '%s' for %s\n", val, a);
        return false;
      }
    }
    return true;
  }
  void usage(const char* prog) const {
    std::printf("usage: %s [options]\n", prog);
    for (const Option& o : m_options)
      std::printf("  --%s%s%s  %s\n", o.long_name.c_str(), o.value_name.empty() ? "" : " ", o.value_name.c_str(),
                  o.help.c_str());
  }

 private:
  struct Option {
    std::string help, long_name, value_name;
    char short_name = 0;
    bool flag = false;
    std::function<bool(const char*)> accept;
  };
  static bool assign(int& v, const char* s) { char* e; v = (int)std::strtol(s, &e, 10); return *e == 0; }
  static bool assign(long& v, const char* s) { char* e; v = std::strtol(s, &e, 10); return *e == 0; }
  static bool assign(float& v, const char* s) { char* e; v = std::strtof(s, &e); return *e == 0; }
  static bool assign(double& v, const char* s) { char* e; v = std::strtod(s, &e); return *e == 0; }
  static bool assign(std::string& v, const char* s) { v = s; return true; }
  static bool assign(const char*& v, const char* s) { v = s; return true; }
  static bool assign(bool& v, const char* s) { v = std::strcmp(s, "0") != 0; return true; }
  std::vector<Option> m_options;
};

class ElapsedTimer {
 public:
  explicit ElapsedTimer(bool precise = false) : m_precise(precise) {}
  bool is_valid() const { return m_valid; }
  void start() {
    m_valid = true;
    m_origin = std::chrono::steady_clock::now();
  }
  int elapsed() const {  // milliseconds since start()
    return (int)std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - m_origin)
        .count();
  }

 private:
  bool m_precise = false;
  bool m_valid = false;
  std::chrono::steady_clock::time_point m_origin{};
};

struct Tracer {
  enum class EventType { StartEvent, EndEvent };
  struct Event {
    EventType etype;
    const char* op;
    long start;
    long end;
  };
  static inline std::vector<Event> events{};
  static inline bool is_trace_on = false;
  static inline long long time_origin = 0;

  static long long now_ms() {
    return (long long)std::chrono::duration_cast<std::chrono::milliseconds>(
               std::chrono::system_clock::now().time_since_epoch())
        .count();
  }
  static void trace_on() {
    time_origin = now_ms();
    is_trace_on = true;
  }
  static void trace_off() { is_trace_on = false; }
  void clear_events() { events.clear(); }

  explicit Tracer(const char* op_) : op(op_) {
    if (is_trace_on) {
      start = now_ms() - time_origin;
      events.push_back({EventType::StartEvent, op, (long)start, (long)end});
    }
  }
  Tracer(const char* op_, bool standalone_) : op(op_), standalone(standalone_) { start = now_ms(); }
  ~Tracer() {
    if (is_trace_on) {
      end = now_ms() - time_origin;
      events.push_back({EventType::EndEvent, op, (long)start, (long)end});
    }
    if (standalone) {
      end = now_ms();
      std::printf("%s tracer end at %lld; started %lld, takes %lld (ms)\n", op, end, start, end - start);
    }
  }
  static void save_events_to_file(const std::string& filename) {
    FILE* f = std::fopen(filename.c_str(), "w");
    if (!f) return;
    for (const Event& e : events) {
      if (e.etype == EventType::StartEvent) std::fprintf(f, "%ld START \"%s\"\n", e.start, e.op);
      else std::fprintf(f, "%ld END \"%s\"\n", e.end, e.op);
    }
    std::fclose(f);
  }

  long long start = 0;
  long long end = -1;
  const char* op;
  bool standalone = false;
};

}  // namespace DArray
