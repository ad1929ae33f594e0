// tvs -- command-line front end with the reference's flags and outputs,
// running the `--compute cuda` backend through libtvs_cuda.so.
//
//   main.rs:21-71     flag handling, default line of sight, DEM set-up
//   config.rs:8-64    flags (--input, --max-line-of-sight, --rings-per-km,
//                     --observer-height, --compute, --output-dir, --scale)
//   input.rs:86-185   .bt reader and scale()
//   compute.rs:101-178 sector loop, running heatmap total, heatmap.png after
//                     every sector
//   output/png.rs:5-37 min/max-normalised 8-bit grey heatmap
//
// Only `--compute cuda` exists in this engine; `cpu` and `vulkan` are the
// reference's other backends and are rejected with an error.  Unlike the
// reference binary (compute.rs:41) the observer height flag is honoured;
// --reference-observer-height pins it to the reference's hard-coded 1.8 m.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "tvs.h"

namespace {

struct Options {
    std::string input;
    long long max_line_of_sight = -1;
    float rings_per_km = 5.0f;
    float observer_height = 1.65f;
    std::string compute = "cuda";
    std::string output_dir = "./";
    double scale = -1.0;
    bool reference_observer_height = false;
    std::string precision = "exact32";
    std::string heatmap = "every-sector";
    std::string surfaces_out;
    int device = 0;
    std::string state_directory;  // empty: the OS state directory (main.rs:63)
    bool cache = true;
};

[[noreturn]] void die(const std::string &msg) {
    std::fprintf(stderr, "Error: %s\n", msg.c_str());
    std::exit(1);
}

// dirs::state_dir() on Linux: $XDG_STATE_HOME if absolute, else $HOME/.local/state.
std::string os_state_directory() {
    const char *x = std::getenv("XDG_STATE_HOME");
    if (x && x[0] == '/') return x;
    const char *h = std::getenv("HOME");
    if (!h || !h[0]) die("Couldn't get the OS's state directory");
    return std::string(h) + "/.local/state";
}

void usage() {
    std::printf(
        "Generate _all_ the viewsheds for a given Digital Elevation Model, therefore the total "
        "viewsheds.\n\n"
        "Usage: tvs --input <PATH> [OPTIONS]\n\n"
        "  --input <PATH>                 the input DEM (.bt)\n"
        "  --max-line-of-sight <METRES>   defaults to one third of the DEM width\n"
        "  --rings-per-km <N>             expected rings per km of band [default: 5]\n"
        "  --observer-height <METRES>     [default: 1.65]\n"
        "  --compute <cuda>               where to run the kernel [default: cuda]\n"
        "  --output-dir <DIR>             heatmap.png goes here [default: ./]\n"
        "  --scale <METRES>               override the DEM point spacing\n"
        "  --reference-observer-height    use the reference binary's hard-coded 1.8 m\n"
        "  --precision <exact32|mixed64|fp64|fp32>  sweep arithmetic [default: exact32]\n"
        "  --state-directory <DIR>        shape cache root [default: the OS state directory]\n"
        "  --no-cache                     neither read nor write the shape cache\n"
        "  --heatmap <every-sector|final> heatmap.png cadence [default: every-sector]\n"
        "  --surfaces-out <PATH>          also write the f32 cumulative surfaces\n"
        "  --device <N>                   CUDA device [default: 0]\n");
}

Options parse(int argc, char **argv) {
    Options o;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto val = [&]() -> std::string {
            if (i + 1 >= argc) die("missing value for " + a);
            return argv[++i];
        };
        if (a == "--help" || a == "-h") { usage(); std::exit(0); }
        else if (a == "--input") o.input = val();
        else if (a == "--max-line-of-sight") o.max_line_of_sight = std::atoll(val().c_str());
        else if (a == "--rings-per-km") o.rings_per_km = std::strtof(val().c_str(), nullptr);
        else if (a == "--observer-height") o.observer_height = std::strtof(val().c_str(), nullptr);
        else if (a == "--compute") o.compute = val();
        else if (a == "--output-dir") o.output_dir = val();
        else if (a == "--scale") o.scale = std::strtod(val().c_str(), nullptr);
        else if (a == "--reference-observer-height") o.reference_observer_height = true;
        else if (a == "--precision") o.precision = val();
        else if (a == "--heatmap") o.heatmap = val();
        else if (a == "--surfaces-out") o.surfaces_out = val();
        else if (a == "--device") o.device = std::atoi(val().c_str());
        else if (a == "--state-directory") o.state_directory = val();
        else if (a == "--no-cache") o.cache = false;
        else die("unknown argument " + a);
    }
    if (o.input.empty()) die("--input is required");
    if (o.compute != "cuda")
        die("this build implements `--compute cuda` only (the reference's cpu and vulkan "
            "backends are not part of it)");
    return o;
}

// ---- .bt (input.rs:86-175) ----------------------------------------------

struct BinaryTerrain {
    uint32_t width = 0, height = 0;
    uint16_t data_size = 0;
    bool is_float = false;
    double left = 0, right = 0, bottom = 0, top = 0;
    std::vector<float> heights;  // f32 whatever the file stores (main.rs:51-56)
};

template <typename T>
T le(const unsigned char *p) {
    T v;
    std::memcpy(&v, p, sizeof v);  // x86-64 and aarch64 hosts are little-endian
    return v;
}

BinaryTerrain read_bt(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) die("cannot open " + path);
    std::vector<unsigned char> raw((std::istreambuf_iterator<char>(f)), {});
    if (raw.size() < 10 || std::memcmp(raw.data(), "binterr1.3", 10) != 0)
        die("Not a Binary Terrain v1.3 file");
    if (raw.size() < 66) die("truncated .bt header");
    BinaryTerrain t;
    const unsigned char *p = raw.data() + 10;
    t.width = le<uint32_t>(p);
    t.height = le<uint32_t>(p + 4);
    t.data_size = le<uint16_t>(p + 8);
    t.is_float = le<uint16_t>(p + 10) != 0;
    t.left = le<double>(p + 18);
    t.right = le<double>(p + 26);
    t.bottom = le<double>(p + 34);
    t.top = le<double>(p + 42);
    const uint64_t n = (uint64_t)t.width * t.height;
    const uint64_t bytes = n * (t.is_float ? 4 : 2);
    if (!t.is_float && t.data_size != 2)
        die("Unsupported `.bt` field value for data size: " + std::to_string(t.data_size));
    if (raw.size() < 256 + bytes) die("truncated .bt elevation data");
    t.heights.resize(n);
    const unsigned char *d = raw.data() + 256;
    for (uint64_t i = 0; i < n; i++)
        t.heights[i] = t.is_float ? le<float>(d + 4 * i) : (float)le<int16_t>(d + 2 * i);
    return t;
}

// input.rs:178-185: geo 0.30 Haversine with the reference's argument order
// (Point::new(top, right): x = top is read as longitude).
double bt_scale(const BinaryTerrain &t) {
    const double r = 6371008.8, deg = 3.14159265358979323846 / 180.0;
    const double lon1 = t.top * deg, lat1 = t.right * deg;
    const double lon2 = t.top * deg, lat2 = t.left * deg;
    const double a = std::pow(std::sin((lat2 - lat1) / 2), 2) +
                     std::cos(lat1) * std::cos(lat2) * std::pow(std::sin((lon2 - lon1) / 2), 2);
    return 2 * r * std::asin(std::sqrt(a)) / t.width;
}

// ---- PNG (output/png.rs:5-37), stored deflate blocks --------------------

uint32_t crc32(const unsigned char *p, size_t n, uint32_t c = 0) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t x = i;
            for (int k = 0; k < 8; k++) x = (x & 1) ? 0xEDB88320u ^ (x >> 1) : x >> 1;
            table[i] = x;
        }
        init = true;
    }
    c = ~c;
    for (size_t i = 0; i < n; i++) c = table[(c ^ p[i]) & 0xFF] ^ (c >> 8);
    return ~c;
}

void put32(std::vector<unsigned char> &v, uint32_t x) {
    for (int s = 24; s >= 0; s -= 8) v.push_back((unsigned char)(x >> s));
}

void chunk(std::vector<unsigned char> &out, const char *type, const std::vector<unsigned char> &d) {
    put32(out, (uint32_t)d.size());
    std::vector<unsigned char> body(type, type + 4);
    body.insert(body.end(), d.begin(), d.end());
    out.insert(out.end(), body.begin(), body.end());
    put32(out, crc32(body.data(), body.size()));
}

bool save_png(const std::vector<float> &data, uint32_t w, uint32_t h, const std::string &path) {
    float mn = INFINITY, mx = -INFINITY;
    for (float v : data) { mn = std::fmin(mn, v); mx = std::fmax(mx, v); }
    const float range = (mx - mn == 0.0f) ? 1.0f : mx - mn;
    std::vector<unsigned char> raw;
    raw.reserve((size_t)(w + 1) * h);
    for (uint32_t y = 0; y < h; y++) {
        raw.push_back(0);  // filter: none
        for (uint32_t x = 0; x < w; x++) {
            float v = (data[(size_t)y * w + x] - mn) / range * 255.0f;
            v = std::fmin(std::fmax(v, 0.0f), 255.0f);
            raw.push_back((unsigned char)v);
        }
    }
    std::vector<unsigned char> z = {0x78, 0x01};
    uint32_t a = 1, b = 0;
    for (unsigned char c : raw) { a = (a + c) % 65521; b = (b + a) % 65521; }
    for (size_t off = 0; off < raw.size() || off == 0; off += 65535) {
        size_t n = std::min<size_t>(65535, raw.size() - off);
        bool last = off + n >= raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back((unsigned char)(n & 0xFF));
        z.push_back((unsigned char)(n >> 8));
        z.push_back((unsigned char)(~n & 0xFF));
        z.push_back((unsigned char)((~n >> 8) & 0xFF));
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + n);
        if (last) break;
    }
    put32(z, (b << 16) | a);
    std::vector<unsigned char> png = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    std::vector<unsigned char> ihdr;
    put32(ihdr, w);
    put32(ihdr, h);
    ihdr.insert(ihdr.end(), {8, 0, 0, 0, 0});  // 8-bit greyscale
    chunk(png, "IHDR", ihdr);
    chunk(png, "IDAT", z);
    chunk(png, "IEND", {});
    std::ofstream f(path, std::ios::binary);
    f.write((const char *)png.data(), (std::streamsize)png.size());
    return (bool)f;
}

void check(int rc, tvs_context *ctx) {
    if (rc != TVS_OK) die(tvs_last_error(ctx));
}

}  // namespace

int main(int argc, char **argv) {
    Options o = parse(argc, argv);
    BinaryTerrain tile = read_bt(o.input);
    const double scale = o.scale > 0 ? o.scale : bt_scale(tile);                 // main.rs:28
    const uint32_t los = o.max_line_of_sight >= 0
                             ? (uint32_t)o.max_line_of_sight
                             : (uint32_t)((double)(tile.width / 3) * scale);    // main.rs:36-38
    tvs_params p{};
    p.width = tile.width;
    p.height = tile.width;  // the reference only reads the header width (main.rs:49)
    if ((uint64_t)tile.width * tile.width > tile.heights.size())
        die("the reference treats the DEM as width x width; this file has fewer rows");
    p.scale = (float)scale;
    p.max_line_of_sight = los;
    p.rings_per_km = o.rings_per_km;
    p.observer_height = o.reference_observer_height ? 1.8f : o.observer_height;
    p.precision = o.precision == "fp64"      ? TVS_PRECISION_FP64
                  : o.precision == "mixed64" ? TVS_PRECISION_MIXED64
                  : o.precision == "fp32"    ? TVS_PRECISION_FP32
                                             : TVS_PRECISION_EXACT32;
    p.sweep_kernel = TVS_SWEEP_ENGINE;
    p.device = o.device;
    std::fprintf(stderr, "Initialising: %ux%u DEM, scale %.3f m, line of sight %u m\n",
                 tile.width, tile.width, scale, los);
    tvs_context *ctx = nullptr;
    check(tvs_create(&p, tile.heights.data(), (uint64_t)tile.width * tile.width, &ctx), nullptr);
    tvs_geometry g;
    tvs_get_geometry(ctx, &g);
    if (o.cache) {  // compute.rs:118-162: load the cached shapes, compute and save the rest
        const std::string dir = o.state_directory.empty() ? os_state_directory() : o.state_directory;
        uint32_t loaded = 0;
        check(tvs_cache_load(ctx, dir.c_str(), &loaded), ctx);
        std::fprintf(stderr, "Shape cache %s/total-viewsheds/%u: %u of 180 sectors loaded\n",
                     dir.c_str(), tile.width, loaded);
        if (loaded < 180) check(tvs_cache_save(ctx, dir.c_str(), 0), ctx);
    }
    std::vector<float> cumulative(g.computable_points_count), total(g.computable_points_count);
    const std::string heatmap = o.output_dir + "/heatmap.png";
    check(tvs_device_reset(ctx), ctx);
    if (o.heatmap == "every-sector") {
        for (uint32_t angle = 0; angle < 180; angle++) {   // compute.rs:106-112
            std::fprintf(stderr, "Running kernel for %u°\n", angle);
            check(tvs_device_run_sectors(ctx, angle, 1), ctx);
            check(tvs_device_finish(ctx), ctx);
            check(tvs_read_surfaces(ctx, nullptr, total.data()), ctx);
            if (!save_png(total, g.tvs_width, g.tvs_height, heatmap)) die("cannot write " + heatmap);
        }
    } else {
        check(tvs_device_run_sectors(ctx, 0, 180), ctx);
        check(tvs_device_finish(ctx), ctx);
    }
    check(tvs_read_surfaces(ctx, cumulative.data(), total.data()), ctx);
    if (!save_png(total, g.tvs_width, g.tvs_height, heatmap)) die("cannot write " + heatmap);
    if (!o.surfaces_out.empty()) {
        std::ofstream f(o.surfaces_out, std::ios::binary);
        f.write((const char *)cumulative.data(), (std::streamsize)(cumulative.size() * 4));
    }
    tvs_destroy(ctx);
    std::fprintf(stderr, "Done: %llu points, heatmap at %s\n",
                 (unsigned long long)g.computable_points_count, heatmap.c_str());
    return 0;
}
