// Host front end: the reference's text handling, restated with buffered I/O and run on all host
// threads.  A file is cut after newline bytes into one range per thread: a word cannot span a
// newline, so every range tokenizes on its own exactly as the sequential reader would.  Results are
// byte-identical to the one-thread restatement (and to the reference): vocabulary entries are
// merged in first-occurrence order, which is the order qsort then sees; a vocabulary that would
// reach ReduceVocab's 21M entries is learned by the sequential path instead.
//
//   ReadWord            PAR_Word2Vec_cpu.cpp:120-144   tokenizer ("</s>" per newline, 98-byte words)
//   LearnVocab...       :253-292                        first-seen order, counts, ReduceVocab at 21M
//   SortVocab           :204-226                        libc qsort of entries 1.., same element layout
//                                                       and comparator, so ties land where the
//                                                       reference's qsort puts them
//   ReadVocab           :301-335                        "word count" lines
//   loadStream          :359-370                        in-vocabulary ids, at most train_words of them
//   saveModel           :721-737                        "%d %d\n", "%s ", "%f " / raw float32
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <fcntl.h>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>
#include <unordered_map>
#include <vector>

#include "../../include/parw2v.h"

namespace {

constexpr int kMaxString = 100;            // MAX_STRING, PAR_Word2Vec_cpu.cpp:31
constexpr long long kReduceAt = 21000000;  // vocab_hash_size * 0.7, :74 and :282

// A FILE-like reader with one byte of push-back and an end-of-file flag that behaves like the
// stdio one the reference polls: it is raised by the read that hits the end.
class Reader {
   public:
    explicit Reader(FILE *f) : f_(f), buf_(1 << 20) {}
    int get() {
        if (pushed_ >= 0) {
            int c = pushed_;
            pushed_ = -1;
            return c;
        }
        if (pos_ == len_) {
            len_ = fread(buf_.data(), 1, buf_.size(), f_);
            pos_ = 0;
            if (len_ == 0) {
                eof_ = true;
                return EOF;
            }
        }
        return (unsigned char) buf_[pos_++];
    }
    void unget(int c) { pushed_ = c; }
    bool eof() const { return eof_; }

   private:
    FILE *f_;
    std::vector<char> buf_;
    size_t pos_ = 0, len_ = 0;
    int pushed_ = -1;
    bool eof_ = false;
};

// ReadWord: returns the word as a C string would hold it (cut at an embedded NUL).
void read_word(Reader &r, std::string &word) {
    char w[kMaxString];
    int a = 0;
    while (!r.eof()) {
        int ch = r.get();
        if (ch == 13) continue;
        if (ch == ' ' || ch == '\t' || ch == '\n') {
            if (a > 0) {
                if (ch == '\n') r.unget(ch);
                break;
            }
            if (ch == '\n') {
                word.assign("</s>");
                return;
            }
            continue;
        }
        w[a] = (char) ch;
        a++;
        if (a >= kMaxString - 1) a--;
    }
    w[a] = 0;
    word.assign(w, strnlen(w, (size_t) a));
}

// The reference's vocab_word layout: qsort sees the same element size and order of fields.
struct VocabWord {
    unsigned int cn;
    char *word;
};

int vocab_compare(const void *a, const void *b) {  // VocabCompare, :199-201
    return (int) (((const VocabWord *) b)->cn - ((const VocabWord *) a)->cn);
}

// ---- parallel tokenizing ----

constexpr uint64_t kMinRange = 1024;  // bytes: smaller files still take more than one range

int host_threads() {
    const unsigned n = std::thread::hardware_concurrency();
    return (int) std::min(32u, std::max(1u, n));
}

// [begin, end) byte ranges that start after a newline byte (the first at 0), in file order.
std::vector<std::pair<uint64_t, uint64_t>> split_at_newlines(int fd, uint64_t size, int parts) {
    std::vector<uint64_t> cuts{0};
    const uint64_t step = std::max<uint64_t>(kMinRange, (size + parts - 1) / std::max(1, parts));
    std::vector<char> buf(1 << 16);
    for (uint64_t want = step; want < size; want += step) {
        uint64_t pos = std::max(want, cuts.back());
        uint64_t cut = size;
        while (pos < size) {  // the first newline at or after pos: the range ends just after it
            const ssize_t got = pread(fd, buf.data(), std::min<uint64_t>(buf.size(), size - pos), (off_t) pos);
            if (got <= 0) break;
            const void *nl = memchr(buf.data(), '\n', (size_t) got);
            if (nl) {
                cut = pos + (uint64_t) ((const char *) nl - buf.data()) + 1;
                break;
            }
            pos += (uint64_t) got;
        }
        if (cut >= size) break;
        if (cut > cuts.back()) cuts.push_back(cut);
    }
    std::vector<std::pair<uint64_t, uint64_t>> ranges;
    for (size_t i = 0; i < cuts.size(); i++) ranges.emplace_back(cuts[i], i + 1 < cuts.size() ? cuts[i + 1] : size);
    return ranges;
}

// ReadWord over a byte range, calling emit(word, length) for every word and "</s>".  A range that
// is not the file's last ends after a newline, so no word is pending at its end; at the end of the
// file a pending word is dropped, as the reference's feof test drops it.
template <class Emit>
bool tokenize_range(int fd, uint64_t begin, uint64_t end, Emit &&emit) {
    std::vector<char> buf(1 << 22);
    char w[kMaxString];
    int a = 0;
    for (uint64_t pos = begin; pos < end;) {
        const ssize_t got = pread(fd, buf.data(), std::min<uint64_t>(buf.size(), end - pos), (off_t) pos);
        if (got <= 0) return false;
        for (ssize_t i = 0; i < got; i++) {
            const char ch = buf[(size_t) i];
            if (ch == 13) continue;
            if (ch == ' ' || ch == '\t' || ch == '\n') {
                if (a > 0) {
                    emit(w, strnlen(w, (size_t) a));
                    a = 0;
                }
                if (ch == '\n') emit("</s>", 4);
                continue;
            }
            w[a] = ch;
            a++;
            if (a >= kMaxString - 1) a--;
        }
        pos += (uint64_t) got;
    }
    return true;
}

// Open-addressing word -> entry table over a byte arena; entries keep first-insertion order.
class WordTable {
   public:
    struct Entry {
        uint64_t off;
        uint32_t len;
        uint64_t count;
    };
    WordTable() { slots_.assign(1 << 12, -1); }
    static uint64_t hash(const char *s, size_t n) {  // FNV-1a, 64 bit
        uint64_t h = 1469598103934665603ULL;
        for (size_t i = 0; i < n; i++) h = (h ^ (unsigned char) s[i]) * 1099511628211ULL;
        return h;
    }
    // index of the word's entry, inserting it (count 0) if absent
    int64_t find_or_add(const char *s, size_t n) {
        if ((entries_.size() + 1) * 2 > slots_.size()) grow();
        size_t i = (size_t) hash(s, n) & (slots_.size() - 1);
        for (;;) {
            const int64_t e = slots_[i];
            if (e < 0) {
                slots_[i] = (int64_t) entries_.size();
                entries_.push_back(Entry{(uint64_t) arena_.size(), (uint32_t) n, 0});
                arena_.insert(arena_.end(), s, s + n);
                return (int64_t) entries_.size() - 1;
            }
            const Entry &x = entries_[(size_t) e];
            if (x.len == n && memcmp(arena_.data() + x.off, s, n) == 0) return e;
            i = (i + 1) & (slots_.size() - 1);
        }
    }
    int64_t find(const char *s, size_t n) const {
        size_t i = (size_t) hash(s, n) & (slots_.size() - 1);
        for (;;) {
            const int64_t e = slots_[i];
            if (e < 0) return -1;
            const Entry &x = entries_[(size_t) e];
            if (x.len == n && memcmp(arena_.data() + x.off, s, n) == 0) return e;
            i = (i + 1) & (slots_.size() - 1);
        }
    }
    std::vector<Entry> &entries() { return entries_; }
    const char *text(const Entry &e) const { return arena_.data() + e.off; }

   private:
    void grow() {
        std::vector<int64_t> next(slots_.size() * 2, -1);
        for (size_t k = 0; k < entries_.size(); k++) {
            size_t i = (size_t) hash(arena_.data() + entries_[k].off, entries_[k].len) & (next.size() - 1);
            while (next[i] >= 0) i = (i + 1) & (next.size() - 1);
            next[i] = (int64_t) k;
        }
        slots_.swap(next);
    }
    std::vector<int64_t> slots_;
    std::vector<Entry> entries_;
    std::vector<char> arena_;
};

int open_sized(const char *path, uint64_t *size) {
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return -1;
    struct stat st;
    if (fstat(fd, &st) != 0) {
        close(fd);
        return -1;
    }
    *size = (uint64_t) st.st_size;
    return fd;
}

}  // namespace

struct parw2v_vocab {
    std::vector<VocabWord> words;  // owned strings
    std::unordered_map<std::string, int> index;
    uint64_t train_words = 0;
    ~parw2v_vocab() {
        for (auto &v : words) free(v.word);
    }
    int add(const std::string &w) {  // AddWordToVocab, :178-196
        size_t n = w.size() + 1 < (size_t) kMaxString ? w.size() + 1 : (size_t) kMaxString;
        char *s = (char *) calloc(n > w.size() + 1 ? n : w.size() + 1, 1);
        memcpy(s, w.data(), w.size());
        words.push_back(VocabWord{0u, s});
        index.emplace(w, (int) words.size() - 1);
        return (int) words.size() - 1;
    }
    void rebuild_index() {
        index.clear();
        index.reserve(words.size() * 2);
        for (size_t i = 0; i < words.size(); i++) index.emplace(std::string(words[i].word), (int) i);
    }
    void reduce(unsigned &min_reduce) {  // ReduceVocab, :229-251 (entry 0 is not protected there)
        size_t k = 0;
        for (size_t i = 0; i < words.size(); i++) {
            if (words[i].cn > min_reduce) words[k++] = words[i];
            else free(words[i].word);
        }
        words.resize(k);
        rebuild_index();
        min_reduce++;
    }
    void sort_and_filter(int min_count) {  // SortVocab, :204-226
        if (words.size() > 1) qsort(&words[1], words.size() - 1, sizeof(VocabWord), vocab_compare);
        std::vector<VocabWord> kept;
        kept.reserve(words.size());
        train_words = 0;
        for (size_t i = 0; i < words.size(); i++) {
            if (words[i].cn < (unsigned) min_count && i != 0) {
                free(words[i].word);
            } else {
                kept.push_back(words[i]);
                train_words += words[i].cn;
            }
        }
        words.swap(kept);
        rebuild_index();
    }
};

// LearnVocabFromTrainFile one word at a time (the reference's order of events, ReduceVocab included)
static int vocab_learn_sequential(const char *train_file, int min_count, parw2v_vocab **out) {
    FILE *f = fopen(train_file, "rb");
    if (!f) return PARW2V_ERR_IO;
    parw2v_vocab *v = new parw2v_vocab();
    v->add("</s>");
    Reader r(f);
    std::string w;
    unsigned min_reduce = 1;
    for (;;) {
        read_word(r, w);
        if (r.eof()) break;
        auto it = v->index.find(w);
        if (it == v->index.end()) v->words[(size_t) v->add(w)].cn = 1;
        else v->words[(size_t) it->second].cn++;
        if ((long long) v->words.size() > kReduceAt) v->reduce(min_reduce);
    }
    fclose(f);
    v->sort_and_filter(min_count);
    *out = v;
    return PARW2V_OK;
}

extern "C" {

int parw2v_vocab_learn(const char *train_file, int min_count, parw2v_vocab **out) {
    if (!train_file || !out) return PARW2V_ERR_ARG;
    *out = nullptr;
    uint64_t size = 0;
    const int fd = open_sized(train_file, &size);
    if (fd < 0) return PARW2V_ERR_IO;
    const auto ranges = split_at_newlines(fd, size, host_threads());
    // count every range on its own thread, words in their first-seen order
    std::vector<WordTable> tables(ranges.size());
    std::vector<char> ok(ranges.size(), 1);
    std::vector<std::thread> pool;
    for (size_t r = 0; r < ranges.size(); r++)
        pool.emplace_back([&, r]() {
            WordTable &t = tables[r];
            ok[r] = tokenize_range(fd, ranges[r].first, ranges[r].second,
                                   [&](const char *w, size_t n) { t.entries()[(size_t) t.find_or_add(w, n)].count++; });
        });
    for (auto &th : pool) th.join();
    close(fd);
    for (char k : ok)
        if (!k) return PARW2V_ERR_IO;
    // merge in range order: a word's index is its first occurrence in the file; "</s>" is entry 0
    WordTable all;
    all.entries()[(size_t) all.find_or_add("</s>", 4)].count = 0;
    for (auto &t : tables) {
        for (const auto &e : t.entries()) all.entries()[(size_t) all.find_or_add(t.text(e), e.len)].count += e.count;
        t = WordTable();
    }
    if ((long long) all.entries().size() > kReduceAt) return vocab_learn_sequential(train_file, min_count, out);
    parw2v_vocab *v = new parw2v_vocab();
    v->words.reserve(all.entries().size());
    for (const auto &e : all.entries()) {
        const std::string w(all.text(e), e.len);
        v->words[(size_t) v->add(w)].cn = (unsigned) e.count;
    }
    v->sort_and_filter(min_count);
    *out = v;
    return PARW2V_OK;
}

int parw2v_vocab_read(const char *vocab_file, int min_count, parw2v_vocab **out) {
    if (!vocab_file || !out) return PARW2V_ERR_ARG;
    *out = nullptr;
    FILE *f = fopen(vocab_file, "rb");
    if (!f) return PARW2V_ERR_IO;
    parw2v_vocab *v = new parw2v_vocab();
    Reader r(f);
    std::string w;
    for (;;) {
        read_word(r, w);
        if (r.eof()) break;
        const int i = v->add(w);
        // fscanf(fin, "%d%c", &cn, &c): skip blanks, an optionally signed decimal, then one byte
        int ch = r.get();
        while (ch == ' ' || ch == '\t' || ch == '\n' || ch == '\r' || ch == '\v' || ch == '\f') ch = r.get();
        long long sign = 1, val = 0;
        bool any = false;
        if (ch == '-' || ch == '+') {
            sign = ch == '-' ? -1 : 1;
            ch = r.get();
        }
        while (ch >= '0' && ch <= '9') {
            val = val * 10 + (ch - '0');
            any = true;
            ch = r.get();
        }
        if (any) v->words[(size_t) i].cn = (unsigned) (sign * val);
        // ch is the %c byte (consumed)
    }
    fclose(f);
    v->sort_and_filter(min_count);
    *out = v;
    return PARW2V_OK;
}

void parw2v_vocab_free(parw2v_vocab *v) { delete v; }

int parw2v_vocab_size(const parw2v_vocab *v) { return v ? (int) v->words.size() : 0; }

uint64_t parw2v_vocab_train_words(const parw2v_vocab *v) { return v ? v->train_words : 0; }

int parw2v_vocab_counts(const parw2v_vocab *v, uint32_t *counts) {
    if (!v || !counts) return PARW2V_ERR_ARG;
    for (size_t i = 0; i < v->words.size(); i++) counts[i] = v->words[i].cn;
    return PARW2V_OK;
}

const char *parw2v_vocab_word(const parw2v_vocab *v, int i) {
    if (!v || i < 0 || (size_t) i >= v->words.size()) return nullptr;
    return v->words[(size_t) i].word;
}

int parw2v_vocab_save(const parw2v_vocab *v, const char *path) {
    if (!v || !path) return PARW2V_ERR_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return PARW2V_ERR_IO;
    for (const auto &e : v->words) fprintf(f, "%s %d\n", e.word, (int) e.cn);
    return fclose(f) == 0 ? PARW2V_OK : PARW2V_ERR_IO;
}

int parw2v_load_stream(const parw2v_vocab *v, const char *train_file, int32_t *tokens, uint64_t capacity,
                       uint64_t *n_tokens) {
    if (!v || !train_file || !n_tokens) return PARW2V_ERR_ARG;
    uint64_t size = 0;
    const int fd = open_sized(train_file, &size);
    if (fd < 0) return PARW2V_ERR_IO;
    // the vocabulary as a word -> id table the threads share read-only
    WordTable ids;
    for (const auto &e : v->words) ids.find_or_add(e.word, strlen(e.word));
    const auto ranges = split_at_newlines(fd, size, host_threads());
    std::vector<std::vector<int32_t>> part(ranges.size());
    std::vector<uint64_t> count(ranges.size(), 0);
    std::vector<char> ok(ranges.size(), 1);
    std::vector<std::thread> pool;
    for (size_t r = 0; r < ranges.size(); r++)
        pool.emplace_back([&, r]() {
            ok[r] = tokenize_range(fd, ranges[r].first, ranges[r].second, [&](const char *w, size_t n) {
                const int64_t id = ids.find(w, n);
                if (id < 0) return;  // out of the vocabulary: skipped (:365)
                if (tokens) part[r].push_back((int32_t) id);
                count[r]++;
            });
        });
    for (auto &th : pool) th.join();
    close(fd);
    for (char k : ok)
        if (!k) return PARW2V_ERR_IO;
    // loadStream keeps at most train_words ids (:361)
    uint64_t n = 0;
    const uint64_t total = v->train_words;
    for (size_t r = 0; r < ranges.size() && n < total; r++) {
        const uint64_t take = std::min<uint64_t>(count[r], total - n);
        if (tokens) {
            if (n + take > capacity) return PARW2V_ERR_CAPACITY;
            memcpy(tokens + n, part[r].data(), sizeof(int32_t) * take);
        }
        n += take;
    }
    *n_tokens = n;
    return PARW2V_OK;
}

int parw2v_save_model(const parw2v_vocab *v, const float *w_in, int size, int binary, const char *path) {
    if (!v || !w_in || size < 1 || !path) return PARW2V_ERR_ARG;
    FILE *fo = fopen(path, "wb");
    if (!fo) return PARW2V_ERR_IO;
    const int V = (int) v->words.size();
    fprintf(fo, "%d %d\n", V, size);
    // blocks of rows are formatted by the host threads ("%s " then "%f " per value, or the raw
    // floats) and written in row order
    const int threads = host_threads();
    const int block = 4096;
    std::vector<std::string> out((size_t) threads);
    bool io_ok = true;
    for (int b0 = 0; b0 < V && io_ok; b0 += block * threads) {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; t++)
            pool.emplace_back([&, t]() {
                std::string &o = out[(size_t) t];
                o.clear();
                char num[64];
                const int lo = b0 + t * block, hi = std::min(V, lo + block);
                for (int a = lo; a < hi; a++) {
                    o += v->words[(size_t) a].word;
                    o += ' ';
                    const float *row = w_in + (size_t) a * size;
                    if (binary) {
                        o.append(reinterpret_cast<const char *>(row), sizeof(float) * (size_t) size);
                    } else {
                        for (int k = 0; k < size; k++) o.append(num, (size_t) snprintf(num, sizeof(num), "%f ", row[k]));
                    }
                    o += '\n';
                }
            });
        for (auto &th : pool) th.join();
        for (const auto &o : out)
            if (!o.empty() && fwrite(o.data(), 1, o.size(), fo) != o.size()) io_ok = false;
    }
    return (fclose(fo) == 0 && io_ok) ? PARW2V_OK : PARW2V_ERR_IO;
}

}  // extern "C"
