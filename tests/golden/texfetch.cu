// Golden-vector generator (test infrastructure): linear-filtered fetches of a
// CUDA 3D float texture built as the reference builds its prefix-sum
// textures (ReconNet4D/DistanceDriven.cu:233-271: a cudaArray of extent
// (nz, ny, nx+1) or (nz, ny+1, nx), border / clamp addressing per dimension,
// cudaFilterModeLinear, unnormalised coordinates).  Reads the table and the
// fetch coordinates from a file, writes the fetched values.  Used by
// make_texfetch_golden.py on a GPU machine to pin the oracle's model of the
// texture unit's weights.
//
//   texfetch in.bin out.bin
//   in.bin : int32 W, H, D, mode0, mode1, mode2 (0 border, 1 clamp), int32 n;
//            float32 table[D][H][W]; float32 coords[n][3] (w, h, d)
//   out.bin: float32 values[n]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

#define CK(x)                                                                              \
    do {                                                                                   \
        cudaError_t e = (x);                                                               \
        if (e != cudaSuccess) {                                                            \
            fprintf(stderr, "%s failed: %s\n", #x, cudaGetErrorString(e));                 \
            return 1;                                                                      \
        }                                                                                  \
    } while (0)

__global__ void fetch(float* out, cudaTextureObject_t t, const float* c, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = tex3D<float>(t, c[3 * i], c[3 * i + 1], c[3 * i + 2]);
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 2;
    int hdr[7];
    if (fread(hdr, 4, 7, f) != 7) return 2;
    const int W = hdr[0], H = hdr[1], D = hdr[2], n = hdr[6];
    std::vector<float> table((size_t)W * H * D), coords((size_t)3 * n), out(n);
    if (fread(table.data(), 4, table.size(), f) != table.size() || fread(coords.data(), 4, coords.size(), f) != coords.size())
        return 2;
    fclose(f);
    cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaArray_t arr;
    CK(cudaMalloc3DArray(&arr, &cd, make_cudaExtent(W, H, D)));
    cudaMemcpy3DParms p;
    memset(&p, 0, sizeof(p));
    p.srcPtr = make_cudaPitchedPtr(table.data(), W * sizeof(float), W, H);
    p.dstArray = arr;
    p.extent = make_cudaExtent(W, H, D);
    p.kind = cudaMemcpyHostToDevice;
    CK(cudaMemcpy3D(&p));
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    for (int k = 0; k < 3; k++) td.addressMode[k] = hdr[3 + k] ? cudaAddressModeClamp : cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureObject_t t;
    CK(cudaCreateTextureObject(&t, &rd, &td, NULL));
    float *dc, *dout;
    CK(cudaMalloc(&dc, coords.size() * 4));
    CK(cudaMalloc(&dout, (size_t)n * 4));
    CK(cudaMemcpy(dc, coords.data(), coords.size() * 4, cudaMemcpyHostToDevice));
    fetch<<<(n + 255) / 256, 256>>>(dout, t, dc, n);
    CK(cudaGetLastError());
    CK(cudaMemcpy(out.data(), dout, (size_t)n * 4, cudaMemcpyDeviceToHost));
    FILE* g = fopen(argv[2], "wb");
    if (!g) return 2;
    fwrite(out.data(), 4, n, g);
    fclose(g);
    return 0;
}
