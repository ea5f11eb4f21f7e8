// Host front end: the reference's text handling, restated with buffered I/O.
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
#include <string>
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

extern "C" {

int parw2v_vocab_learn(const char *train_file, int min_count, parw2v_vocab **out) {
    if (!train_file || !out) return PARW2V_ERR_ARG;
    *out = nullptr;
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
    FILE *f = fopen(train_file, "rb");
    if (!f) return PARW2V_ERR_IO;
    Reader r(f);
    std::string w;
    uint64_t n = 0;
    const uint64_t total = v->train_words;
    while (!r.eof() && n < total) {  // loadStream, :361
        read_word(r, w);
        if (r.eof()) break;
        auto it = v->index.find(w);
        if (it == v->index.end()) continue;
        if (tokens) {
            if (n >= capacity) {
                fclose(f);
                return PARW2V_ERR_CAPACITY;
            }
            tokens[n] = it->second;
        }
        n++;
    }
    fclose(f);
    *n_tokens = n;
    return PARW2V_OK;
}

int parw2v_save_model(const parw2v_vocab *v, const float *w_in, int size, int binary, const char *path) {
    if (!v || !w_in || size < 1 || !path) return PARW2V_ERR_ARG;
    FILE *fo = fopen(path, "wb");
    if (!fo) return PARW2V_ERR_IO;
    const int V = (int) v->words.size();
    fprintf(fo, "%d %d\n", V, size);
    std::vector<char> line;
    for (int a = 0; a < V; a++) {
        fprintf(fo, "%s ", v->words[(size_t) a].word);
        const float *row = w_in + (size_t) a * size;
        if (binary) {
            fwrite(row, sizeof(float), (size_t) size, fo);
        } else {
            for (int b = 0; b < size; b++) fprintf(fo, "%f ", row[b]);
        }
        fprintf(fo, "\n");
    }
    return fclose(fo) == 0 ? PARW2V_OK : PARW2V_ERR_IO;
}

}  // extern "C"
