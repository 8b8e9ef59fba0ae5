#include "decoder.h"
namespace idx2g
{
int dataset_open(device_ctx*, const params&, dataset_handle** out) { *out = nullptr; return OptionNotSupported; }
int dataset_output_grid(const dataset_handle*, const params&, grid*) { return OptionNotSupported; }
int dataset_decode(device_ctx*, dataset_handle*, const params&, void*, size_t, bool, double*) { return OptionNotSupported; }
void dataset_close(dataset_handle*) {}
}
