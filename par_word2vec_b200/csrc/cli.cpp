// parw2v: drop-in command line for PAR_Word2Vec_cpu / PAR_Word2Vec_gpu_{text,graph}.
//
// Accepts the reference's flags (PAR_Word2Vec_cpu.cpp:786-818; the GPU binaries add -gamma and
// -max-num-sen, PAR_Word2Vec_gpu_text.cu:1083-1086), reads the corpus and vocabulary exactly as
// the reference does, trains on the GPU through libparw2v's C ABI and writes the reference's
// output formats: the -output embedding file (text "%f " or binary), -save-vocab, and the
// "PAR_Word2Vec_gpu_time" file holding "Elapsed <seconds>" (device time of training, as the GPU
// reference measures it).  Extra flags: -mode det|plain|batched|batched_bf16 (default
// batched_bf16), -device <n>, -seed <n>, -attraction sequential|window.
// Accepted for compatibility and ignored: -threads (the GPU replaces the OpenMP threads; -mode det
// reproduces the reference at -threads 1), -disk, -gamma, -max-num-sen (no sentence-count limit).
// Unlike the reference, every failure exits with a non-zero status and a message.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "parw2v.h"

static int arg_pos(const char *s, int argc, char **argv) {
    for (int a = 1; a < argc; a++)
        if (!strcmp(s, argv[a])) return a;
    return -1;
}

static void usage() {
    printf("parallel word2vec (sgns) on NVIDIA B200 -- drop-in for PAR_Word2Vec_cpu / _gpu\n\n");
    printf("Options (as the reference): -train <file> -output <file> -size <int> -window <int>\n");
    printf("  -sample <float> -negative <int> -threads <int> -iter <int> -min-count <int> -alpha <float>\n");
    printf("  -debug <int> -binary <int> -save-vocab <file> -read-vocab <file> -batch-size <int> -disk\n");
    printf("  -gamma <int> -max-num-sen <int>   (GPU reference flags, accepted and ignored)\n");
    printf("Extra: -mode det|plain|batched|batched_bf16 (default batched_bf16) -device <int> -seed <int>\n");
    printf("       -attraction sequential|window\n");
}

static int die(int rc, const char *what, parw2v_ctx *ctx) {
    fprintf(stderr, "parw2v: %s failed: %s (%s)\n", what, parw2v_strerror(rc), parw2v_last_error(ctx));
    return 1;
}

int main(int argc, char **argv) {
    if (argc == 1) {
        usage();
        return 0;
    }
    std::string train_file, output_file, save_vocab, read_vocab;
    parw2v_config cfg;
    memset(&cfg, 0, sizeof(cfg));
    // the reference CPU defaults (PAR_Word2Vec_cpu.cpp:64-69)
    cfg.size = 100;
    cfg.window = 5;
    cfg.negative = 5;
    cfg.batch_size = 24;
    cfg.iter = 5;
    cfg.alpha = 0.025f;
    cfg.sample = 1e-3f;
    cfg.mode = PARW2V_MODE_BATCHED_BF16;
    int min_count = 5, binary = 0, debug = 2;
    int i;
    if ((i = arg_pos("-size", argc, argv)) > 0 && i + 1 < argc) cfg.size = atoi(argv[i + 1]);
    if ((i = arg_pos("-train", argc, argv)) > 0 && i + 1 < argc) train_file = argv[i + 1];
    if ((i = arg_pos("-save-vocab", argc, argv)) > 0 && i + 1 < argc) save_vocab = argv[i + 1];
    if ((i = arg_pos("-read-vocab", argc, argv)) > 0 && i + 1 < argc) read_vocab = argv[i + 1];
    if ((i = arg_pos("-debug", argc, argv)) > 0 && i + 1 < argc) debug = atoi(argv[i + 1]);
    if ((i = arg_pos("-binary", argc, argv)) > 0 && i + 1 < argc) binary = atoi(argv[i + 1]);
    if ((i = arg_pos("-alpha", argc, argv)) > 0 && i + 1 < argc) cfg.alpha = (float) atof(argv[i + 1]);
    if ((i = arg_pos("-output", argc, argv)) > 0 && i + 1 < argc) output_file = argv[i + 1];
    if ((i = arg_pos("-window", argc, argv)) > 0 && i + 1 < argc) cfg.window = atoi(argv[i + 1]);
    if ((i = arg_pos("-sample", argc, argv)) > 0 && i + 1 < argc) cfg.sample = (float) atof(argv[i + 1]);
    if ((i = arg_pos("-negative", argc, argv)) > 0 && i + 1 < argc) cfg.negative = atoi(argv[i + 1]);
    if ((i = arg_pos("-iter", argc, argv)) > 0 && i + 1 < argc) cfg.iter = atoi(argv[i + 1]);
    if ((i = arg_pos("-min-count", argc, argv)) > 0 && i + 1 < argc) min_count = atoi(argv[i + 1]);
    if ((i = arg_pos("-batch-size", argc, argv)) > 0 && i + 1 < argc) cfg.batch_size = atoi(argv[i + 1]);
    if ((i = arg_pos("-device", argc, argv)) > 0 && i + 1 < argc) cfg.device = atoi(argv[i + 1]);
    if ((i = arg_pos("-seed", argc, argv)) > 0 && i + 1 < argc) cfg.seed = strtoull(argv[i + 1], nullptr, 10);
    if ((i = arg_pos("-mode", argc, argv)) > 0 && i + 1 < argc) {
        const char *m = argv[i + 1];
        if (!strcmp(m, "det")) cfg.mode = PARW2V_MODE_DET;
        else if (!strcmp(m, "plain")) cfg.mode = PARW2V_MODE_PLAIN;
        else if (!strcmp(m, "batched")) cfg.mode = PARW2V_MODE_BATCHED;
        else if (!strcmp(m, "batched_bf16")) cfg.mode = PARW2V_MODE_BATCHED_BF16;
        else {
            fprintf(stderr, "parw2v: unknown -mode %s\n", m);
            return 2;
        }
    }
    if ((i = arg_pos("-attraction", argc, argv)) > 0 && i + 1 < argc)
        cfg.attraction = !strcmp(argv[i + 1], "window") ? PARW2V_ATTRACT_WINDOW : PARW2V_ATTRACT_SEQUENTIAL;
    if (train_file.empty() && read_vocab.empty()) {
        fprintf(stderr, "parw2v: -train is required\n");
        return 2;
    }
    if (debug > 0) {
        printf("number of iterations: %d\n", cfg.iter);
        printf("hidden size: %d\n", cfg.size);
        printf("number of negative samples: %d\n", cfg.negative);
        printf("window size: %d\n", cfg.window);
        printf("batch size: %d\n", cfg.batch_size);
        printf("starting learning rate: %.5f\n", cfg.alpha);
        printf("starting training using file: %s\n\n", train_file.c_str());
    }

    parw2v_vocab *vocab = nullptr;
    int rc = read_vocab.empty() ? parw2v_vocab_learn(train_file.c_str(), min_count, &vocab)
                                : parw2v_vocab_read(read_vocab.c_str(), min_count, &vocab);
    if (rc) return die(rc, read_vocab.empty() ? "reading the training file" : "reading the vocabulary", nullptr);
    const int V = parw2v_vocab_size(vocab);
    if (debug > 0) {
        printf("Vocab size: %d\n", V);
        printf("Words in train file: %llu\n", (unsigned long long) parw2v_vocab_train_words(vocab));
    }
    if (!save_vocab.empty() && (rc = parw2v_vocab_save(vocab, save_vocab.c_str()))) return die(rc, "-save-vocab", nullptr);
    if (output_file.empty()) {
        parw2v_vocab_free(vocab);
        return 0;
    }
    // loadStream keeps at most train_words ids (PAR_Word2Vec_cpu.cpp:361): one pass into that much
    uint64_t n = 0;
    const uint64_t cap = parw2v_vocab_train_words(vocab);
    std::vector<int32_t> tokens(cap ? cap : 1);
    if ((rc = parw2v_load_stream(vocab, train_file.c_str(), tokens.data(), tokens.size(), &n)))
        return die(rc, "loading the corpus", nullptr);
    std::vector<uint32_t> counts((size_t) V);
    parw2v_vocab_counts(vocab, counts.data());

    parw2v_ctx *ctx = nullptr;
    if ((rc = parw2v_create(&cfg, &ctx))) return die(rc, "creating the GPU context", nullptr);
    if ((rc = parw2v_set_vocab(ctx, counts.data(), V))) return die(rc, "building the unigram table", ctx);
    if ((rc = parw2v_init_weights(ctx))) return die(rc, "InitNet", ctx);
    if ((rc = parw2v_set_corpus(ctx, tokens.data(), n))) return die(rc, "uploading the corpus", ctx);
    parw2v_stats st;
    if ((rc = parw2v_train(ctx, &st))) return die(rc, "training", ctx);
    const double seconds = (st.kernel_ms + st.pack_ms) / 1000.0;
    if (debug > 0)
        printf("\ntrained %llu words in %.3f s (%.2f M words/sec)\n", (unsigned long long) st.words, seconds,
               seconds > 0 ? st.words / seconds / 1e6 : 0.0);
    FILE *ft = fopen("PAR_Word2Vec_gpu_time", "w");
    if (ft) {
        fprintf(ft, "Elapsed %.2lf", seconds);
        fclose(ft);
    }
    std::vector<float> w_in((size_t) V * cfg.size);
    if ((rc = parw2v_get_weights(ctx, w_in.data(), nullptr))) return die(rc, "reading the weights", ctx);
    if ((rc = parw2v_save_model(vocab, w_in.data(), cfg.size, binary, output_file.c_str())))
        return die(rc, "-output", ctx);
    parw2v_destroy(ctx);
    parw2v_vocab_free(vocab);
    return 0;
}
