// cli.cpp -- the `cuSZp` command-line tool: same flags, output lines and file
// formats as the reference's examples/cuSZp.cpp (usage :23-61, parsing :64-148,
// relative bound :176-210, timing :237-261, report :264-303, writes :306-317).
// The relative error bound is reduced on the device (cuSZp_rel_error_bound)
// with the reference's float arithmetic instead of a serial host loop.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cuda_runtime.h>
#include <cuSZp.h>

static void usage()
{
    printf("cuSZp: A GPU error-bounded lossy compressor for floating-point data (B200 build)\n\n");
    printf("Usage:\n");
    printf("  ./cuSZp -i [oriFilePath] -t [dataType] -m [encodingMode] -d [dim] [dim_z] [dim_y] [dim_x] "
           "-eb [errorBoundMode] [errorBound] -x [cmpFilePath] -o [decFilePath]\n\n");
    printf("Options:\n");
    printf("  -i  [oriFilePath]    Path to the input file containing the original data\n");
    printf("  -t  [dataType]       f32 | f64\n");
    printf("  -m  [encodingMode]   fixed | plain | outlier\n");
    printf("  -d  [dim]            1 | 2 [dim_z] [dim_y] [dim_x] | 3 [dim_z] [dim_y] [dim_x] (dim_x fastest)\n");
    printf("  -eb [errorBoundMode] [errorBound]   abs | rel, e.g. -eb rel 1e-4\n");
    printf("  -x  [cmpFilePath]    Path to the compressed output file (optional)\n");
    printf("  -o  [decFilePath]    Path to the decompressed output file (optional)\n");
    exit(EXIT_FAILURE);
}

int main(int argc, char* argv[])
{
    char oriFilePath[640] = {0}, cmpFilePath[640] = {0}, decFilePath[640] = {0};
    cuszp_dim_t processingDim = CUSZP_DIM_1D;
    cuszp_type_t dataType = CUSZP_TYPE_FLOAT;
    cuszp_mode_t encodingMode = CUSZP_MODE_PLAIN;
    char errorBoundMode[4] = {0};
    float errorBound = 0.0f;
    uint3 dims = {0, 0, 0};

    if (argc == 1 || (argc == 2 && (!strcmp(argv[1], "-h") || !strcmp(argv[1], "--help")))) usage();
    for (int i = 1; i < argc; i++) {
        if (!strcmp(argv[i], "-i") && i + 1 < argc) {
            strncpy(oriFilePath, argv[++i], sizeof(oriFilePath) - 1);
        } else if (!strcmp(argv[i], "-t") && i + 1 < argc) {
            ++i;
            if (!strcmp(argv[i], "f32")) dataType = CUSZP_TYPE_FLOAT;
            else if (!strcmp(argv[i], "f64")) dataType = CUSZP_TYPE_DOUBLE;
            else { printf("Error: Unsupported data type. Use 'f32' or 'f64'.\n"); exit(EXIT_FAILURE); }
        } else if (!strcmp(argv[i], "-m") && i + 1 < argc) {
            ++i;
            if (!strcmp(argv[i], "plain")) encodingMode = CUSZP_MODE_PLAIN;
            else if (!strcmp(argv[i], "outlier")) encodingMode = CUSZP_MODE_OUTLIER;
            else if (!strcmp(argv[i], "fixed")) encodingMode = CUSZP_MODE_FIXED;
            else { printf("Error: Unsupported encoding mode. Use 'fixed', 'plain', or 'outlier'.\n"); exit(EXIT_FAILURE); }
        } else if (!strcmp(argv[i], "-d") && i + 1 < argc) {
            processingDim = (cuszp_dim_t)atoi(argv[i + 1]);
            if (processingDim == 2 || processingDim == 3) {
                if (i + 4 >= argc) { printf("Error: Missing dimension sizes for 2D/3D processing.\n"); exit(EXIT_FAILURE); }
                dims.z = (unsigned)atoi(argv[i + 2]);
                dims.y = (unsigned)atoi(argv[i + 3]);
                dims.x = (unsigned)atoi(argv[i + 4]);
                i += 4;
            } else if (processingDim == 1) {
                i += 1;
            } else {
                printf("Error: Unsupported processing dimension. Use 1, 2, or 3.\n"); exit(EXIT_FAILURE);
            }
        } else if (!strcmp(argv[i], "-eb") && i + 2 < argc) {
            strncpy(errorBoundMode, argv[i + 1], sizeof(errorBoundMode) - 1);
            if (strcmp(errorBoundMode, "rel") && strcmp(errorBoundMode, "abs")) {
                printf("Error: Unsupported error bound mode. Use 'rel' or 'abs'.\n"); exit(EXIT_FAILURE);
            }
            errorBound = (float)atof(argv[i + 2]);
            i += 2;
        } else if (!strcmp(argv[i], "-x") && i + 1 < argc) {
            strncpy(cmpFilePath, argv[++i], sizeof(cmpFilePath) - 1);
        } else if (!strcmp(argv[i], "-o") && i + 1 < argc) {
            strncpy(decFilePath, argv[++i], sizeof(decFilePath) - 1);
        } else {
            printf("Error: Unrecognized option '%s'.\n", argv[i]);
            exit(EXIT_FAILURE);
        }
    }
    if (strlen(oriFilePath) == 0 || errorBound == 0.0f) { printf("Error: Missing required arguments.\n"); exit(EXIT_FAILURE); }

    TimingGPU timer_GPU;
    const size_t esize = dataType == CUSZP_TYPE_FLOAT ? sizeof(float) : sizeof(double);
    size_t nbEle = 0, cmpSize = 0;
    int status = 0;
    void* oriData = dataType == CUSZP_TYPE_FLOAT ? (void*)readFloatData_Yafan(oriFilePath, &nbEle, &status)
                                                 : (void*)readDoubleData_Yafan(oriFilePath, &nbEle, &status);
    if (!oriData || status) { fprintf(stderr, "Error: cannot read %s\n", oriFilePath); return 1; }
    if (processingDim != CUSZP_DIM_1D && nbEle != (size_t)dims.x * (size_t)dims.y * (size_t)dims.z) {
        fprintf(stderr, "Error: The number of elements in the original data does not match the dimensions\n");
        return 1;
    }
    void* decData = malloc(nbEle * esize + 1);

    // The stream can exceed the input size on incompressible data; size the
    // device buffer for the worst case instead of nbEle * sizeof(T).
    const size_t cap = cuSZp_max_compressed_size(nbEle, processingDim, dims, dataType, encodingMode);
    unsigned char* cmpBytes = (unsigned char*)malloc(cap + 1);
    void *d_oriData, *d_decData;
    unsigned char* d_cmpBytes;
    cudaMalloc(&d_oriData, nbEle * esize + 16);
    cudaMemcpy(d_oriData, oriData, nbEle * esize, cudaMemcpyHostToDevice);
    cudaMalloc(&d_decData, nbEle * esize + 16);
    cudaMalloc((void**)&d_cmpBytes, cap + 16);
    cudaMemset(d_decData, 0, nbEle * esize);

    if (!strcmp(errorBoundMode, "rel")) {
        float eb_abs = 0.0f;
        if (cuSZp_rel_error_bound(d_oriData, nbEle, dataType, errorBound, &eb_abs, 0) != CUSZP_SUCCESS) {
            fprintf(stderr, "Error: value range reduction failed\n");
            return 1;
        }
        errorBound = eb_abs;
    }

    cudaStream_t stream;
    cudaStreamCreate(&stream);
    for (int i = 0; i < 10; i++)
        cuSZp_compress(d_oriData, d_cmpBytes, nbEle, &cmpSize, errorBound, processingDim, dims, dataType, encodingMode, stream);

    timer_GPU.StartCounter();
    cuSZp_compress(d_oriData, d_cmpBytes, nbEle, &cmpSize, errorBound, processingDim, dims, dataType, encodingMode, stream);
    const float cmpTime = timer_GPU.GetCounter();

    // Round trip of exactly cmpSize bytes through the host checks the reported size.
    unsigned char* cmpBytes_dup = (unsigned char*)malloc(cmpSize + 1);
    cudaMemcpy(cmpBytes_dup, d_cmpBytes, cmpSize, cudaMemcpyDeviceToHost);
    cudaMemset(d_cmpBytes, 0, cap);
    cudaMemcpy(d_cmpBytes, cmpBytes_dup, cmpSize, cudaMemcpyHostToDevice);

    timer_GPU.StartCounter();
    cuSZp_decompress(d_decData, d_cmpBytes, nbEle, cmpSize, errorBound, processingDim, dims, dataType, encodingMode, stream);
    const float decTime = timer_GPU.GetCounter();

    const double mib = nbEle * (double)esize / 1024.0 / 1024.0;
    printf("cuSZp finished!\n");
    printf("cuSZp compression   end-to-end speed: %f GB/s\n", mib / cmpTime);
    printf("cuSZp decompression end-to-end speed: %f GB/s\n", mib / decTime);
    printf("cuSZp compression ratio: %f\n\n", mib / (cmpSize / 1024.0 / 1024.0));

    cudaMemcpy(decData, d_decData, nbEle * esize, cudaMemcpyDeviceToHost);
    size_t not_bound = 0, over_eb = 0;
    for (size_t i = 0; i < nbEle; i++) {
        double a, b;
        if (dataType == CUSZP_TYPE_FLOAT) { a = ((float*)oriData)[i]; b = ((float*)decData)[i]; }
        else { a = ((double*)oriData)[i]; b = ((double*)decData)[i]; }
        const double err = fabs(a - b);
        if (dataType == CUSZP_TYPE_FLOAT ? (double)fabsf((float)a - (float)b) > errorBound * 1.1 : err > errorBound * 1.1) not_bound++;
        if (err > (double)errorBound) over_eb++;
    }
    if (!not_bound) printf("\033[0;32mPass error check!\033[0m\n");
    else printf("\033[0;31mFail error check! Exceeding data count: %zu\033[0m\n", not_bound);
    printf("FP64 check: %zu of %zu values beyond eb (reference tolerance 1.1*eb)\n", over_eb, nbEle);

    if (strlen(cmpFilePath) > 0) {
        cudaMemcpy(cmpBytes, d_cmpBytes, cmpSize, cudaMemcpyDeviceToHost);
        writeByteData_Yafan(cmpBytes, cmpSize, cmpFilePath, &status);
    }
    if (strlen(decFilePath) > 0) {
        if (dataType == CUSZP_TYPE_FLOAT) writeFloatData_inBytes_Yafan((float*)decData, nbEle, decFilePath, &status);
        else writeDoubleData_inBytes_Yafan((double*)decData, nbEle, decFilePath, &status);
    }

    free(oriData); free(decData); free(cmpBytes); free(cmpBytes_dup);
    cudaFree(d_oriData); cudaFree(d_decData); cudaFree(d_cmpBytes);
    cudaStreamDestroy(stream);
    return not_bound ? 2 : 0;
}
