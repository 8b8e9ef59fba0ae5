// idx2g_app: command-line front end with the reference idx2App's options
// (Applications/idx2App.cpp:17-212), running the CUDA library through its C ABI.
//
//   idx2g_app --encode Name-Field-[X-Y-Z]-Float32.raw --num_levels 2 --tolerance 1e-3
//             [--brick_size 32 32 32] [--bricks_per_chunk N] [--chunks_per_file N]
//             [--files_per_dir N] [--bit_planes_per_chunk N] [--out_dir D]
//             [--name N --field F --dims X Y Z --type float32|float64]
//   idx2g_app --decode D/Name/Field.idx2 [--first x y z --last x y z]
//             [--downsampling a b c] [--tolerance t] [--in_dir D] [--out_dir D]
//             [--out_file F] [--dry] [--brick_map] [--parallel]
//
// --parallel selects the reference's thread-pool decode (Applications/idx2App.cpp:56,
// Core/idx2ParallelDecode.cpp:484), whose output equals its sequential decode's; every decode
// here runs in parallel on the GPU, so the option is accepted and changes nothing.
#include "../../include/idx2g.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

namespace
{

int find(int argc, char** argv, const char* opt)
{
  for (int i = 1; i < argc; ++i)
    if (strcmp(argv[i], opt) == 0)
      return i;
  return -1;
}

bool opt_str(int argc, char** argv, const char* opt, std::string* v)
{
  int i = find(argc, argv, opt);
  if (i < 0 || i + 1 >= argc)
    return false;
  *v = argv[i + 1];
  return true;
}

bool opt_int(int argc, char** argv, const char* opt, int* v)
{
  std::string s;
  if (!opt_str(argc, argv, opt, &s))
    return false;
  *v = atoi(s.c_str());
  return true;
}

bool opt_dbl(int argc, char** argv, const char* opt, double* v)
{
  std::string s;
  if (!opt_str(argc, argv, opt, &s))
    return false;
  *v = atof(s.c_str());
  return true;
}

bool opt_v3(int argc, char** argv, const char* opt, int v[3])
{
  int i = find(argc, argv, opt);
  if (i < 0 || i + 3 >= argc)
    return false;
  for (int k = 0; k < 3; ++k)
    v[k] = atoi(argv[i + 1 + k]);
  return true;
}

std::string parent_path(const std::string& p)
{
  size_t k = p.find_last_of('/');
  if (k == std::string::npos)
    return p;
  return p.substr(0, k);
}

std::string file_name(const std::string& p)
{
  size_t k = p.find_last_of('/');
  return k == std::string::npos ? p : p.substr(k + 1);
}

int die(const char* what, int code)
{
  fprintf(stderr, "%s: %s (%d)\n", what, idx2g_error_string(code), code);
  return 1;
}

int do_encode(int argc, char** argv)
{
  idx2g_params p;
  idx2g_params_init(&p);
  std::string in;
  opt_str(argc, argv, "--encode", &in);
  // Core/DataSet.cpp:48 StrToMetaData: "Name-Field-[X-Y-Z]-Type.raw"
  char name[64] = {}, field[64] = {}, type[16] = {};
  int dims[3] = { 0, 0, 0 };
  std::string fn = file_name(in);
  if (sscanf(fn.c_str(), "%63[^-]-%63[^-]-[%d-%d-%d]-%15[^.]", name, field, &dims[0], &dims[1], &dims[2],
             type) != 6)
  {
    std::string s;
    if (!opt_str(argc, argv, "--name", &s))
    {
      fprintf(stderr, "Provide --name\n");
      return 1;
    }
    snprintf(name, sizeof name, "%s", s.c_str());
    if (!opt_str(argc, argv, "--field", &s))
    {
      fprintf(stderr, "Provide --field\n");
      return 1;
    }
    snprintf(field, sizeof field, "%s", s.c_str());
    if (!opt_v3(argc, argv, "--dims", dims))
    {
      fprintf(stderr, "Provide --dims\n");
      return 1;
    }
    if (!opt_str(argc, argv, "--type", &s))
    {
      fprintf(stderr, "Provide --type (float32 or float64)\n");
      return 1;
    }
    snprintf(type, sizeof type, "%s", s.c_str());
  }
  type[0] = (char)tolower(type[0]);
  if (strcmp(type, "float32") && strcmp(type, "float64"))
  {
    fprintf(stderr, "Unsupported type\n");
    return 1;
  }
  snprintf(p.name, sizeof p.name, "%s", name);
  snprintf(p.field, sizeof p.field, "%s", field);
  for (int k = 0; k < 3; ++k)
    p.dims[k] = dims[k];
  p.dtype = strcmp(type, "float32") == 0 ? IDX2G_FLOAT32 : IDX2G_FLOAT64;
  opt_v3(argc, argv, "--brick_size", p.brick_dims);
  opt_int(argc, argv, "--num_levels", &p.num_levels);
  opt_dbl(argc, argv, "--tolerance", &p.tolerance);
  if (p.tolerance <= 0)
  {
    p.tolerance = p.dtype == IDX2G_FLOAT32 ? 1.1920928955078125e-07 : 2.220446049250313e-16;
    printf("tolerance = %.16f (machine epsilon)\n", p.tolerance);
  }
  opt_int(argc, argv, "--bit_planes_per_chunk", &p.bit_planes_per_chunk);
  opt_int(argc, argv, "--bit_planes_per_file", &p.bit_planes_per_file);
  opt_int(argc, argv, "--bricks_per_chunk", &p.bricks_per_chunk);
  opt_int(argc, argv, "--chunks_per_file", &p.chunks_per_file);
  opt_int(argc, argv, "--files_per_dir", &p.files_per_dir);
  std::string od;
  if (opt_str(argc, argv, "--out_dir", &od))
    snprintf(p.out_dir, sizeof p.out_dir, "%s", od.c_str());

  int e = idx2g_check_params(&p);
  if (e)
    return die("parameters", e);
  size_t n = (size_t)p.dims[0] * (size_t)p.dims[1] * (size_t)p.dims[2];
  size_t bytes = n * (p.dtype == IDX2G_FLOAT32 ? 4 : 8);
  std::vector<unsigned char> raw(bytes);
  FILE* fp = fopen(in.c_str(), "rb");
  if (!fp || fread(raw.data(), 1, bytes, fp) != bytes)
  {
    fprintf(stderr, "cannot read %s\n", in.c_str());
    return 1;
  }
  fclose(fp);
  idx2g_ctx* ctx = nullptr;
  e = idx2g_ctx_create(0, nullptr, &ctx);
  if (e)
    return die("context", e);
  auto t0 = std::chrono::steady_clock::now();
  idx2g_encode_info info;
  e = idx2g_encode(ctx, &p, raw.data(), 0, &info);
  auto t1 = std::chrono::steady_clock::now();
  idx2g_ctx_destroy(ctx);
  if (e)
    return die("encode", e);
  printf("kernel time             = %f ms\n", info.kernel_ms);
  printf("total time              = %f seconds\n", std::chrono::duration<double>(t1 - t0).count());
  return 0;
}

int do_decode(int argc, char** argv)
{
  idx2g_params p;
  idx2g_params_init(&p);
  std::string in;
  opt_str(argc, argv, "--decode", &in);
  snprintf(p.input_file, sizeof p.input_file, "%s", in.c_str());
  if (find(argc, argv, "--first") >= 0 || find(argc, argv, "--last") >= 0)
  {
    if (!opt_v3(argc, argv, "--first", p.first) || !opt_v3(argc, argv, "--last", p.last))
    {
      fprintf(stderr, "Provide --first and --last\n");
      return 1;
    }
    p.has_extent = 1;
  }
  opt_v3(argc, argv, "--downsampling", p.downsampling);
  opt_dbl(argc, argv, "--tolerance", &p.decode_tolerance);
  std::string s;
  if (opt_str(argc, argv, "--in_dir", &s))
    snprintf(p.in_dir, sizeof p.in_dir, "%s", s.c_str());
  else
  {
    // Applications/idx2App.cpp:43-49
    std::string parent = parent_path(in);
    std::string d = parent_path(parent);
    if (d == parent)
      d = "./";
    snprintf(p.in_dir, sizeof p.in_dir, "%s", d.c_str());
  }
  std::string out_dir = ".", out_file;
  opt_str(argc, argv, "--out_dir", &out_dir);
  bool have_out_file = opt_str(argc, argv, "--out_file", &out_file);
  bool dry = find(argc, argv, "--dry") >= 0;

  idx2g_ctx* ctx = nullptr;
  int e = idx2g_ctx_create(0, nullptr, &ctx);
  if (e)
    return die("context", e);
  idx2g_dataset* ds = nullptr;
  e = idx2g_dataset_open(ctx, &p, &ds);
  if (e)
  {
    idx2g_ctx_destroy(ctx);
    return die("open", e);
  }
  if (find(argc, argv, "--brick_map") >= 0)
  {
    // Applications/idx2App.cpp:51-53: the HashMap output mode, written to "bricks" in the
    // working directory (Core/idx2Decode.cpp:477)
    double kms = 0;
    auto t0 = std::chrono::steady_clock::now();
    e = idx2g_decode_brick_map(ctx, ds, &p, "bricks", &kms);
    auto t1 = std::chrono::steady_clock::now();
    idx2g_dataset_close(ds);
    idx2g_ctx_destroy(ctx);
    if (e)
      return die("decode", e);
    printf("kernel time         = %f ms\n", kms);
    printf("total decode time   = %f\n", std::chrono::duration<double>(t1 - t0).count());
    return 0;
  }
  int from[3], dims[3], strd[3];
  idx2g_output_grid(ds, &p, from, dims, strd);
  char name[64], field[64];
  int vd[3], dt, nl;
  double tol;
  long long resident;
  idx2g_dataset_info(ds, name, field, vd, &dt, &nl, &tol, &resident);
  size_t n = (size_t)dims[0] * (size_t)dims[1] * (size_t)dims[2];
  size_t es = dt == IDX2G_FLOAT32 ? 4 : 8;
  std::vector<unsigned char> out(n * es);
  auto t0 = std::chrono::steady_clock::now();
  double kms = 0;
  e = idx2g_decode(ctx, ds, &p, out.data(), out.size(), 0, &kms);
  auto t1 = std::chrono::steady_clock::now();
  idx2g_dataset_close(ds);
  idx2g_ctx_destroy(ctx);
  if (e)
    return die("decode", e);
  printf("kernel time         = %f ms\n", kms);
  printf("total decode time   = %f\n", std::chrono::duration<double>(t1 - t0).count());
  if (dry)
    return 0;
  // Core/idx2Decode.cpp:344-345: "<out_dir>/<Name>-<Field>-[X-Y-Z]-<type>-tolerance-%f.raw"
  char path[1024];
  if (have_out_file)
    snprintf(path, sizeof path, "%s/%s", out_dir.c_str(), out_file.c_str());
  else
    snprintf(path, sizeof path, "%s/%s-%s-[%d-%d-%d]-%s-tolerance-%f.raw", out_dir.c_str(), name, field,
             dims[0], dims[1], dims[2], dt == IDX2G_FLOAT32 ? "float32" : "float64", p.decode_tolerance);
  FILE* fp = fopen(path, "wb");
  if (!fp || fwrite(out.data(), 1, out.size(), fp) != out.size())
  {
    fprintf(stderr, "cannot write %s\n", path);
    return 1;
  }
  fclose(fp);
  printf("writing output volume to %s\n", path);
  return 0;
}

} // namespace

int main(int argc, char** argv)
{
  if (find(argc, argv, "--encode") >= 0)
    return do_encode(argc, argv);
  if (find(argc, argv, "--decode") >= 0)
    return do_decode(argc, argv);
  fprintf(stderr, "Provide either --encode or --decode\n"
                  "Example 1: --encode /Users/abc/Miranda-Density-[384-384-256]-Float64.raw\n"
                  "Example 2: --decode Miranda/Density.idx2\n");
  return 1;
}
