// TEST INFRASTRUCTURE ONLY - part of the oracle, never linked into the
// product library.
//
// A small stand-in for the TTG (Template Task Graph) runtime header, written
// for this project so that the reference Barnes-Hut solver's unmodified
// sources compile and run on a machine without TTG/PaRSEC/MADNESS/MPI.
// It supports exactly the subset the reference uses on one rank:
//
//   Edge<K, V>, edges(...), make_tt(fn, ins, outs, name), make_aggregator,
//   Aggregator<V>, send<i>/sendk<i> from inside a task, in<0>()->send/sendk
//   and invoke() from outside, set_keymap (ignored), make_graph_executable
//   (no-op), fence, initialize/execute/finalize, default_execution_context()
//   with rank 0 of 1, print, and the declarations the multi-rank code needs
//   to compile (SplitMetadataDescriptor, madness::archive::wrap).
//
// Tasks run on a thread pool. Its size is TTG_NUM_THREADS when set, else
// every CPU this process may run on. fence() blocks until every task
// submitted so far, and every task those spawned, has finished.
#pragma once

#include <sched.h>
#include <sys/uio.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <deque>
#include <functional>
#include <iostream>
#include <unordered_map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <tuple>
#include <type_traits>
#include <typeinfo>
#include <utility>
#include <vector>

namespace madness::archive {
// Only named by serialize() members that are never instantiated on one rank.
template <typename T>
struct Wrapped {
  T* ptr;
  std::size_t n;
};
template <typename T>
inline Wrapped<T> wrap(T* ptr, std::size_t n) {
  return {ptr, n};
}
}  // namespace madness::archive

namespace ttg {

// Customisation point the multi-rank exchange specialises; unused here.
template <typename T>
struct SplitMetadataDescriptor;

namespace shim {

class Pool {
 public:
  static Pool& get() {
    static Pool pool;
    return pool;
  }

  void start(int nthreads) {
    std::lock_guard<std::mutex> lock(m_);
    if (!workers_.empty()) return;
    if (nthreads <= 0) nthreads = default_threads();
    stopping_ = false;
    for (int i = 0; i < nthreads; ++i) workers_.emplace_back([this] { loop(); });
  }

  void stop() {
    {
      std::lock_guard<std::mutex> lock(m_);
      stopping_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
    workers_.clear();
  }

  void submit(std::function<void()> f) {
    start(0);
    {
      std::lock_guard<std::mutex> lock(m_);
      ++pending_;
      queue_.push_back(std::move(f));
    }
    cv_.notify_one();
  }

  void wait_idle() {
    std::unique_lock<std::mutex> lock(m_);
    idle_.wait(lock, [this] { return pending_ == 0; });
    if (error_) {
      auto e = error_;
      error_ = nullptr;
      std::rethrow_exception(e);
    }
  }

  int size() const { return static_cast<int>(workers_.size()); }

  ~Pool() {
    if (!workers_.empty()) stop();
  }

 private:
  static int default_threads() {
    if (const char* s = std::getenv("TTG_NUM_THREADS")) {
      int n = std::atoi(s);
      if (n > 0) return n;
    }
    cpu_set_t set;
    if (sched_getaffinity(0, sizeof(set), &set) == 0) return std::max(1, CPU_COUNT(&set));
    return std::max(1u, std::thread::hardware_concurrency());
  }

  void loop() {
    for (;;) {
      std::function<void()> task;
      {
        std::unique_lock<std::mutex> lock(m_);
        cv_.wait(lock, [this] { return stopping_ || !queue_.empty(); });
        if (queue_.empty()) return;  // stopping and drained
        task = std::move(queue_.front());
        queue_.pop_front();
      }
      try {
        task();
      } catch (...) {
        std::lock_guard<std::mutex> lock(m_);
        if (!error_) error_ = std::current_exception();
      }
      {
        std::lock_guard<std::mutex> lock(m_);
        if (--pending_ == 0) idle_.notify_all();
      }
    }
  }

  std::mutex m_;
  std::condition_variable cv_, idle_;
  std::deque<std::function<void()>> queue_;
  std::vector<std::thread> workers_;
  std::size_t pending_ = 0;
  bool stopping_ = false;
  std::exception_ptr error_;
};

// A type-erased output terminal of the running task: where send<i> goes.
struct OutSlot {
  const std::type_info* key_type;
  const std::type_info* value_type;  // typeid(void) for key-only edges
  std::function<void(const void* key, const void* value)> deliver;
};

inline thread_local const std::vector<OutSlot>* current_outs = nullptr;

}  // namespace shim

struct World {
  int rank() const { return 0; }
  int size() const { return 1; }
};
inline World default_execution_context() { return {}; }

inline void initialize(int, char**, int nthreads = -1) { shim::Pool::get().start(nthreads); }
inline void execute() {}
inline void fence() { shim::Pool::get().wait_idle(); }
inline void finalize() { shim::Pool::get().wait_idle(); }

template <typename... Ts>
void print(const Ts&... ts) {
  static std::mutex m;
  std::lock_guard<std::mutex> lock(m);
  ((std::cout << ts << ' '), ...);
  std::cout << '\n';
}

class TTBase {
 public:
  virtual ~TTBase() = default;
  void make_executable() {}
};

template <typename... TTs>
void make_graph_executable(TTs*...) {}

// An edge: the consumers registered by the TTs that take it as input.
template <typename K, typename V = void>
class Edge {
 public:
  using key_type = K;
  using value_type = V;
  using consumer_t =
      std::conditional_t<std::is_void_v<V>, std::function<void(const K&)>, std::function<void(const K&, const std::conditional_t<std::is_void_v<V>, int, V>&)>>;
  struct Impl {
    std::mutex m;
    std::vector<consumer_t> consumers;
  };
  Edge() : impl(std::make_shared<Impl>()) {}
  explicit Edge(const char*) : Edge() {}
  std::shared_ptr<Impl> impl;

  void add_consumer(consumer_t c) {
    std::lock_guard<std::mutex> lock(impl->m);
    impl->consumers.push_back(std::move(c));
  }
  std::vector<consumer_t> consumers() const {
    std::lock_guard<std::mutex> lock(impl->m);
    return impl->consumers;
  }
};

template <typename... Es>
auto edges(Es&&... es) {
  return std::make_tuple(std::decay_t<Es>(es)...);
}

// The values delivered to one key of an aggregator edge.
template <typename V>
class Aggregator {
 public:
  Aggregator() = default;
  explicit Aggregator(std::vector<V> v) : values_(std::move(v)) {}
  auto begin() const { return values_.begin(); }
  auto end() const { return values_.end(); }
  std::size_t size() const { return values_.size(); }

 private:
  std::vector<V> values_;
};

template <typename K, typename V, typename F>
struct AggregatorEdge {
  Edge<K, V> edge;
  F target;
};

template <typename K, typename V, typename F>
auto make_aggregator(const Edge<K, V>& e, F&& target) {
  return AggregatorEdge<K, V, std::decay_t<F>>{e, std::forward<F>(target)};
}

namespace shim {

template <typename E>
struct InTraits;

template <typename K, typename V>
struct InTraits<Edge<K, V>> {
  using key_type = K;
  using value_type = V;
};

template <typename K, typename V, typename F>
struct InTraits<AggregatorEdge<K, V, F>> {
  using key_type = K;
  using value_type = V;
};

template <typename E>
OutSlot make_out_slot(const E& e) {
  using K = typename E::key_type;
  using V = typename E::value_type;
  OutSlot s;
  s.key_type = &typeid(K);
  if constexpr (std::is_void_v<V>) {
    s.value_type = &typeid(void);
    s.deliver = [e](const void* k, const void*) {
      for (auto& c : e.consumers()) c(*static_cast<const K*>(k));
    };
  } else {
    s.value_type = &typeid(V);
    s.deliver = [e](const void* k, const void* v) {
      for (auto& c : e.consumers()) c(*static_cast<const K*>(k), *static_cast<const V*>(v));
    };
  }
  return s;
}

}  // namespace shim

// A template task: fn(key[, value]) runs as a pool task for every key
// delivered on its input edge.
template <typename InEdge, typename Fn, typename OutTuple>
class TT : public TTBase {
 public:
  using K = typename shim::InTraits<InEdge>::key_type;
  using V = typename shim::InTraits<InEdge>::value_type;

  // Input terminal used to seed the graph from outside any task.
  class InTerminal {
   public:
    explicit InTerminal(TT* tt) : tt_(tt) {}
    template <typename Val>
    void send(const K& key, Val&& v) {
      tt_->submit(key, std::decay_t<Val>(std::forward<Val>(v)));
    }
    void sendk(const K& key) { tt_->submit_key(key); }

   private:
    TT* tt_;
  };

  TT(Fn fn, InEdge in, OutTuple outs, std::string name)
      : state_(std::make_shared<State>(std::move(fn), std::move(name))), terminal_(this) {
    std::apply([this](auto&... e) { (state_->outs.push_back(shim::make_out_slot(e)), ...); }, outs);
    connect(in);
  }

  template <std::size_t I>
  InTerminal* in() {
    static_assert(I == 0, "the stand-in runtime supports one input edge per TT");
    return &terminal_;
  }

  template <typename Keymap>
  void set_keymap(Keymap&&) {}

  void invoke(const K& key) { submit_key(key); }

  template <typename Val>
  void submit(const K& key, Val value) {
    auto st = state_;
    shim::Pool::get().submit([st, key, value = std::move(value)]() { st->run(key, value); });
  }
  void submit_key(const K& key) {
    auto st = state_;
    shim::Pool::get().submit([st, key]() { st->run_key(key); });
  }

 private:
  struct State {
    State(Fn f, std::string n) : fn(std::move(f)), name(std::move(n)) {}
    Fn fn;
    std::string name;
    std::vector<shim::OutSlot> outs;
    // aggregator inputs only: values gathered so far, per key
    std::mutex agg_m;
    std::unordered_map<K, std::vector<std::conditional_t<std::is_void_v<V>, int, V>>> pending;

    template <typename Arg>
    void run(const K& key, const Arg& v) {
      const auto* saved = shim::current_outs;
      shim::current_outs = &outs;
      fn(key, v);
      shim::current_outs = saved;
    }
    void run_key(const K& key) {
      const auto* saved = shim::current_outs;
      shim::current_outs = &outs;
      fn(key);
      shim::current_outs = saved;
    }
  };

  template <typename K2, typename V2>
  void connect(Edge<K2, V2>& e) {
    auto st = state_;
    if constexpr (std::is_void_v<V2>) {
      e.add_consumer([st](const K2& k) {
        shim::Pool::get().submit([st, k]() { st->run_key(k); });
      });
    } else {
      e.add_consumer([st](const K2& k, const V2& v) {
        shim::Pool::get().submit([st, k, v]() { st->run(k, v); });
      });
    }
  }

  template <typename K2, typename V2, typename F>
  void connect(AggregatorEdge<K2, V2, F>& a) {
    auto st = state_;
    F target = a.target;
    a.edge.add_consumer([st, target](const K2& k, const V2& v) {
      std::vector<V2> ready;
      {
        std::lock_guard<std::mutex> lock(st->agg_m);
        auto& vec = st->pending[k];
        vec.push_back(v);
        if (vec.size() < static_cast<std::size_t>(target(k))) return;
        ready = std::move(vec);
        st->pending.erase(k);
      }
      shim::Pool::get().submit([st, k, ready = std::move(ready)]() mutable {
        Aggregator<V2> agg(std::move(ready));
        st->run(k, agg);
      });
    });
  }

  std::shared_ptr<State> state_;
  InTerminal terminal_;
};

template <typename Fn, typename InEdge, typename... OutEdges, typename... Rest>
auto make_tt(Fn&& fn, std::tuple<InEdge> ins, std::tuple<OutEdges...> outs, const char* name, Rest&&...) {
  using TTt = TT<InEdge, std::decay_t<Fn>, std::tuple<OutEdges...>>;
  return std::make_unique<TTt>(std::forward<Fn>(fn), std::get<0>(ins), std::move(outs), name);
}

template <std::size_t I, typename K, typename V>
void send(const K& key, V&& value) {
  using D = std::decay_t<V>;
  const auto* outs = shim::current_outs;
  if (outs == nullptr || I >= outs->size()) throw std::logic_error("ttg::send outside a task or to a missing output");
  const shim::OutSlot& s = (*outs)[I];
  if (*s.key_type != typeid(K) || *s.value_type != typeid(D)) throw std::logic_error("ttg::send type mismatch");
  const D copy(std::forward<V>(value));
  s.deliver(&key, &copy);
}

template <std::size_t I, typename K>
void sendk(const K& key) {
  const auto* outs = shim::current_outs;
  if (outs == nullptr || I >= outs->size()) throw std::logic_error("ttg::sendk outside a task or to a missing output");
  const shim::OutSlot& s = (*outs)[I];
  if (*s.key_type != typeid(K) || *s.value_type != typeid(void)) throw std::logic_error("ttg::sendk type mismatch");
  s.deliver(&key, nullptr);
}

}  // namespace ttg
