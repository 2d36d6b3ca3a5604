// worker.cpp -- `femm_gpu --worker` (alias `--motor-worker`): a long-running process that
// serves batch transactions named by job envelopes on standard input.
//
// Wire behaviour (the reference's streaming worker, gpu_solver/src/app/motor_worker.cpp:
// 33-191): each input line is an envelope {"session", "sequence", "request_path",
// "response_path", "request_sha256"}; each envelope gets exactly one status line
// {"session", "sequence", "request_sha256", "exit_code", "prepare_seconds",
// "prepare_begin_seconds", "prepare_end_seconds", "solve_begin_seconds",
// "solve_end_seconds", "error"} on standard output, in input order.  The refusal texts, the
// order in which they are checked, the 32-item transaction cap and the session / sequence
// rule are the reference's, so a client sees the same answers.
//
// Design:
//  * admission -- a table of rules run in order on one envelope line; the first rule that
//    fails names the refusal.  An admitted transaction has its request parsed (neutral
//    gpu_femm_magnetostatic_batch_v1 or a gpu_femm_motor_batch_v* protocol) and every
//    artifact it names read and hashed; artifacts not yet resident are parsed and their
//    plans built on the host, up to four at a time;
//  * look-ahead -- the thread that owns CUDA solves transaction n while one asynchronous
//    task reads and admits line n + 1, so at most one admitted transaction waits beside
//    the one being solved;
//  * ledger -- the session / sequence state: an admitted transaction runs only when it is
//    the next number of the current session (the first fixes the session); a refused one
//    still uses up its number when it was the next one, without GPU work;
//  * resident artifacts -- plans and postprocess masks stay on the device across
//    transactions, at most kResidentArtifacts, the least recently used evicted first.  An
//    artifact file is re-read and re-hashed for every transaction that names it, so a
//    changed file fails that transaction's items exactly as a one-shot --batch would.
#include "worker.h"

#include "json.h"

#include <algorithm>
#include <future>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <stdexcept>
#include <system_error>
#include <thread>

namespace fgcli
{
namespace
{

using Clock = std::chrono::steady_clock;
constexpr size_t kTransactionItems = 32;  // items per transaction, however many envelopes
constexpr size_t kResidentArtifacts = 32; // artifacts kept on the device between transactions
constexpr size_t kLoaderThreads = 4;      // artifacts parsed / planned side by side

// ---------------------------------------------------------------- resident artifacts
class ResidentArtifacts
{
public:
  std::set<ArtifactKey> Keys() const
  {
    std::lock_guard<std::mutex> hold(mutex_);
    std::set<ArtifactKey> keys;
    for (const auto &entry : plans_)
      keys.insert(entry.first);
    return keys;
  }

  // Takes in what admission staged and returns the artifacts `names` resolve to for this
  // transaction: a failed staged check (a stale or unreadable file) for this transaction
  // only, else the resident plan.  Used artifacts become the most recent; beyond the
  // capacity the least recent artifacts outside this transaction are freed.
  ArtifactCache ViewFor(const ArtifactCache &staged, const std::vector<ArtifactKey> &names)
  {
    std::lock_guard<std::mutex> hold(mutex_);
    ArtifactCache view;
    for (const auto &entry : staged) {
      if (entry.second->status != 0)
        view.insert(entry);
      else
        plans_[entry.first] = entry.second;
    }
    for (const ArtifactKey &key : names) {
      if (view.count(key))
        continue;
      const auto it = plans_.find(key);
      if (it == plans_.end())
        continue;
      view.insert(*it);
      stamp_[key] = ++clock_;
    }
    while (plans_.size() > kResidentArtifacts) {
      const ArtifactKey *oldest = nullptr;
      uint64_t oldest_stamp = UINT64_MAX;
      for (const auto &entry : plans_) {
        if (view.count(entry.first))
          continue;
        const uint64_t s = stamp_[entry.first];
        if (s < oldest_stamp) {
          oldest_stamp = s;
          oldest = &entry.first;
        }
      }
      if (!oldest)
        break; // everything left is in use by this transaction
      const ArtifactKey victim = *oldest;
      stamp_.erase(victim);
      plans_.erase(victim);
    }
    return view;
  }

private:
  mutable std::mutex mutex_;
  ArtifactCache plans_;
  std::map<ArtifactKey, uint64_t> stamp_;
  uint64_t clock_ = 0;
};

// The distinct (artifact path, SHA-256) pairs a transaction names, in item order.
std::vector<ArtifactKey> ArtifactsNamed(const StreamTransaction &t)
{
  std::vector<ArtifactKey> keys;
  auto note = [&keys](const std::string &path, const std::string &sha) {
    ArtifactKey key{path, sha};
    if (std::find(keys.begin(), keys.end(), key) == keys.end())
      keys.push_back(std::move(key));
  };
  if (t.motor)
    for (const fgio::MotorBatchItem &item : t.motor_batch.items)
      note(item.request.mesh_artifact_path, item.request.mesh_artifact_sha256);
  else
    for (const fgio::BatchItem &item : t.neutral.items)
      note(item.request.mesh_artifact_path, item.request.mesh_artifact_sha256);
  return keys;
}

// ---------------------------------------------------------------- admission
struct Admission {
  const std::string &line;
  const std::string &executable;
  StreamTransaction &txn;
  fgio::Json envelope;
  std::string request_bytes;
  std::string own_message; // a rule's own refusal text (the request readers' messages)
};

bool EnvelopeHasExactFields(Admission &a)
{
  std::string ignored;
  return fgio::ParseJson(a.line, &a.envelope, &ignored) &&
         fgio::HasExactly(a.envelope, {"session", "sequence", "request_path", "response_path", "request_sha256"},
                          &ignored);
}

bool EnvelopeIdentity(Admission &a)
{
  using K = fgio::Json::Kind;
  std::string ignored;
  const fgio::Json *fields[5] = {a.envelope.get("session", K::String, &ignored),
                                 a.envelope.get("sequence", K::Number, &ignored),
                                 a.envelope.get("request_path", K::String, &ignored),
                                 a.envelope.get("response_path", K::String, &ignored),
                                 a.envelope.get("request_sha256", K::String, &ignored)};
  if (std::any_of(std::begin(fields), std::end(fields), [](const fgio::Json *f) { return f == nullptr; }))
    return false;
  // Both digests are lower-case hex; the number is read (and reported) before its range check.
  if (!fgio::IsSha256Hex(fields[0]->text) || !fgio::IsSha256Hex(fields[4]->text) ||
      !fgio::AsInt32(*fields[1], &a.txn.sequence) || a.txn.sequence < 1)
    return false;
  a.txn.session = fields[0]->text;
  a.txn.request_path = fields[2]->text;
  a.txn.response_path = fields[3]->text;
  a.txn.request_sha256 = fields[4]->text;
  return true;
}

bool OutputPathIsSafe(Admission &a)
{
  const StreamTransaction &t = a.txn;
  return !t.request_path.empty() && !t.response_path.empty() && !SameFile(t.response_path, t.request_path) &&
         !SameFile(t.response_path, a.executable);
}

bool RequestBytesMatch(Admission &a)
{
  return ReadFile(a.txn.request_path, &a.request_bytes) && fgio::Sha256Hex(a.request_bytes) == a.txn.request_sha256;
}

bool RequestParses(Admission &a)
{
  // A gpu_femm_motor_batch_v* protocol takes the motor reader; anything else the neutral one.
  fgio::Json probe;
  std::string ignored;
  if (fgio::ParseJson(a.request_bytes, &probe, &ignored) && probe.is(fgio::Json::Kind::Object)) {
    const auto it = probe.members.find("protocol");
    a.txn.motor = it != probe.members.end() && it->second.is(fgio::Json::Kind::String) &&
                  it->second.text.compare(0, 22, "gpu_femm_motor_batch_v") == 0;
  }
  return a.txn.motor ? fgio::ParseMotorBatchRequestText(a.request_bytes, &a.txn.motor_batch, &a.own_message)
                     : fgio::ParseBatchRequestText(a.request_bytes, &a.txn.neutral, &a.own_message);
}

bool TransactionBounded(Admission &a)
{
  const size_t items = a.txn.motor ? a.txn.motor_batch.items.size() : a.txn.neutral.items.size();
  return items <= kTransactionItems;
}

bool ResponseSparesArtifacts(Admission &a)
{
  for (const ArtifactKey &key : ArtifactsNamed(a.txn))
    if (SameFile(a.txn.response_path, key.first))
      return false;
  return true;
}

struct AdmissionRule {
  const char *refusal; // nullptr: the rule supplies its own message
  bool (*holds)(Admission &);
};

// In the reference's order (motor_worker.cpp:38-82): a line failing several rules is
// refused with the same text.
const AdmissionRule kAdmissionRules[] = {
    {"invalid stream job envelope", EnvelopeHasExactFields},
    {"invalid stream job identity", EnvelopeIdentity},
    {"unsafe stream output path", OutputPathIsSafe},
    {"stream request SHA-256 mismatch", RequestBytesMatch},
    {nullptr, RequestParses},
    {"stream transaction exceeds 32 items", TransactionBounded},
    {"stream response would overwrite an artifact", ResponseSparesArtifacts},
};

// Runs fn(0 .. count-1) on up to `width` threads (thread w takes w, w + width, ...); a
// stride whose thread cannot be started runs on the caller.
void ForEachStrided(size_t count, size_t width, const std::function<void(size_t)> &fn)
{
  width = std::max<size_t>(1, std::min(width, count));
  auto stride = [&](size_t first) {
    for (size_t i = first; i < count; i += width)
      fn(i);
  };
  std::vector<std::thread> threads;
  std::vector<size_t> unstarted;
  for (size_t w = 1; w < width; ++w) {
    try {
      threads.emplace_back(stride, w);
    } catch (const std::system_error &) {
      unstarted.push_back(w);
    }
  }
  stride(0);
  for (size_t w : unstarted)
    stride(w);
  for (std::thread &t : threads)
    t.join();
}

// Reads every artifact the transaction names.  A resident one is only re-read and
// re-hashed (its plan stays); a failed check is staged so that this transaction's items
// fail with the one-shot adapter's message.  The others are parsed and planned on the host.
void StageArtifacts(StreamTransaction &t, const Options &opt, const std::set<ArtifactKey> &resident)
{
  const std::vector<ArtifactKey> keys = ArtifactsNamed(t);
  std::vector<std::shared_ptr<Prepared>> staged(keys.size());
  ForEachStrided(keys.size(), kLoaderThreads, [&](size_t i) {
    const ArtifactKey &key = keys[i];
    auto p = std::make_shared<Prepared>();
    if (resident.count(key)) {
      std::string bytes;
      if (!ReadFile(key.first, &bytes)) {
        p->status = FG_INPUT_IO;
        p->error = "cannot open mesh artifact";
      } else if (fgio::Sha256Hex(bytes) != key.second) {
        p->status = FG_INVALID_ARGUMENT;
        p->error = "mesh artifact SHA mismatch";
      } else {
        return; // unchanged: the resident plan serves it
      }
    } else {
      Prepare(key.first, key.second, opt, p.get());
      PreparePlanOnHost(p.get(), opt);
    }
    staged[i] = std::move(p);
  });
  for (size_t i = 0; i < keys.size(); ++i)
    if (staged[i])
      t.staged[keys[i]] = std::move(staged[i]);
}

std::unique_ptr<StreamTransaction> Admit(const std::string &line, const std::string &executable,
                                         const Options &opt, const ResidentArtifacts &resident)
{
  auto txn = std::make_unique<StreamTransaction>();
  txn->prepare_begin = Clock::now();
  try {
    Admission a{line, executable, *txn, {}, {}, {}};
    for (const AdmissionRule &rule : kAdmissionRules) {
      if (!rule.holds(a)) {
        txn->refusal = rule.refusal ? rule.refusal : a.own_message;
        break;
      }
    }
    if (txn->refusal.empty()) {
      StageArtifacts(*txn, opt, resident.Keys());
      txn->prepare_seconds = std::chrono::duration<double>(Clock::now() - txn->prepare_begin).count();
    }
  } catch (const std::exception &e) {
    txn->refusal = e.what();
  }
  txn->prepare_end = Clock::now();
  return txn;
}

// ---------------------------------------------------------------- session / sequence
class SequenceLedger
{
public:
  bool IsNext(const StreamTransaction &t) const
  {
    return (session_.empty() || session_ == t.session) && t.sequence == last_ + 1;
  }
  void Consume(const StreamTransaction &t)
  {
    session_ = t.session;
    last_ = t.sequence;
  }

private:
  std::string session_;
  int32_t last_ = 0;
};

void WriteStatus(std::ostream &out, const StreamTransaction &t, int exit_code, const std::string &error,
                 Clock::time_point origin, Clock::time_point solve_begin, Clock::time_point solve_end)
{
  auto at = [origin](Clock::time_point p) { return std::chrono::duration<double>(p - origin).count(); };
  out << std::setprecision(17) << "{\"session\":\"" << fgio::Escape(t.session) << "\",\"sequence\":" << t.sequence
      << ",\"request_sha256\":\"" << t.request_sha256 << "\",\"exit_code\":" << exit_code
      << ",\"prepare_seconds\":" << t.prepare_seconds << ",\"prepare_begin_seconds\":" << at(t.prepare_begin)
      << ",\"prepare_end_seconds\":" << at(t.prepare_end) << ",\"solve_begin_seconds\":" << at(solve_begin)
      << ",\"solve_end_seconds\":" << at(solve_end) << ",\"error\":\"" << fgio::Escape(error) << "\"}"
      << std::endl;
}

} // namespace

int ServeStream(std::istream &in, std::ostream &out, const Options &opt, const std::string &executable,
                const TransactionSolver &solve)
{
  const Clock::time_point origin = Clock::now();
  ResidentArtifacts resident;
  SequenceLedger ledger;
  // Only the look-ahead task reads `in`; it returns nullptr at end of input.
  auto admit_next = [&]() {
    return std::async(std::launch::async, [&]() -> std::unique_ptr<StreamTransaction> {
      std::string line;
      if (!std::getline(in, line))
        return nullptr;
      return Admit(line, executable, opt, resident);
    });
  };
  std::future<std::unique_ptr<StreamTransaction>> ahead = admit_next();
  for (;;) {
    std::unique_ptr<StreamTransaction> txn = ahead.get();
    if (!txn)
      break;
    const Clock::time_point solve_begin = Clock::now();
    std::string error = txn->refusal;
    int exit_code = 1;
    const bool next = ledger.IsNext(*txn);
    const bool runs = next && txn->refusal.empty();
    if (next)
      ledger.Consume(*txn); // a refused transaction uses up its number too, without GPU work
    else if (txn->refusal.empty())
      error = "stream session or submission sequence mismatch";
    // Adopt this transaction's staged artifacts before the look-ahead asks what is resident.
    ArtifactCache view;
    if (runs)
      view = resident.ViewFor(txn->staged, ArtifactsNamed(*txn));
    txn->staged.clear();
    ahead = admit_next();
    if (runs) {
      try {
        bool pass = false;
        const std::string text = solve(*txn, &view, &pass);
        if (PublishAtomically(txn->response_path, text))
          exit_code = pass ? 0 : 1;
        else
          error = "could not atomically publish response";
      } catch (const std::exception &e) {
        error = e.what();
      }
    }
    WriteStatus(out, *txn, exit_code, error, origin, solve_begin, Clock::now());
  }
  return 0;
}

} // namespace fgcli
