// utility.cpp -- raw binary file I/O of include/cuSZp/cuSZp_utility.h (the CLI's
// input/output helpers; same names and status convention as the reference's
// src/cuSZp_utility.cu).  Files hold little-endian values; on a little-endian
// host the bytes are read and written as they are.
#include "../../include/cuSZp/cuSZp_utility.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace {

constexpr int kOk = 0;
constexpr int kFileError = 1;

bool host_is_little_endian()
{
    const uint16_t probe = 1;
    unsigned char b;
    std::memcpy(&b, &probe, 1);
    return b == 1;
}

unsigned char* read_all(const char* path, size_t* len, int* status)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        std::printf("Failed to open input file. %s\n", path);
        *status = kFileError;
        *len = 0;
        return nullptr;
    }
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    unsigned char* buf = (unsigned char*)std::malloc(sz > 0 ? (size_t)sz : 1);
    const size_t got = buf ? std::fread(buf, 1, (size_t)sz, f) : 0;
    std::fclose(f);
    *len = got;
    *status = buf ? kOk : kFileError;
    return buf;
}

template <typename T>
T* read_values(const char* path, size_t* nbEle, int* status, bool swap)
{
    size_t len = 0;
    unsigned char* bytes = read_all(path, &len, status);
    *nbEle = len / sizeof(T);
    if (!bytes) return nullptr;
    if (swap) {
        for (size_t i = 0; i < *nbEle; i++) {
            unsigned char* p = bytes + i * sizeof(T);
            for (size_t a = 0, b = sizeof(T) - 1; a < b; a++, b--) { unsigned char t = p[a]; p[a] = p[b]; p[b] = t; }
        }
    }
    return reinterpret_cast<T*>(bytes);
}

void write_all(const void* data, size_t len, const char* path, int* status)
{
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        std::printf("Failed to open output file. %s\n", path);
        *status = kFileError;
        return;
    }
    std::fwrite(data, 1, len, f);
    std::fclose(f);
    *status = kOk;
}

template <typename T>
void write_values_le(const T* data, size_t n, const char* path, int* status)
{
    if (host_is_little_endian()) { write_all(data, n * sizeof(T), path, status); return; }
    unsigned char* bytes = (unsigned char*)std::malloc(n * sizeof(T) + 1);
    for (size_t i = 0; i < n; i++)
        for (size_t k = 0; k < sizeof(T); k++)
            bytes[i * sizeof(T) + k] = reinterpret_cast<const unsigned char*>(data + i)[sizeof(T) - 1 - k];
    write_all(bytes, n * sizeof(T), path, status);
    std::free(bytes);
}

}  // namespace

void symTransform_2bytes(unsigned char data[2]) { unsigned char t = data[0]; data[0] = data[1]; data[1] = t; }

void symTransForm_4Bytes(unsigned char data[4])
{
    unsigned char t = data[0]; data[0] = data[3]; data[3] = t;
    t = data[1]; data[1] = data[2]; data[2] = t;
}

void symTransform_8bytes(unsigned char data[8])
{
    for (int a = 0, b = 7; a < b; a++, b--) { unsigned char t = data[a]; data[a] = data[b]; data[b] = t; }
}

void convertUShortArrayToBytes(unsigned short* states, size_t stateLength, unsigned char* bytes)
{
    for (size_t i = 0; i < stateLength; i++) { bytes[2 * i] = (unsigned char)states[i]; bytes[2 * i + 1] = (unsigned char)(states[i] >> 8); }
}

void convertUIntArrayToBytes(unsigned int* states, size_t stateLength, unsigned char* bytes)
{
    for (size_t i = 0; i < stateLength; i++)
        for (int k = 0; k < 4; k++) bytes[4 * i + k] = (unsigned char)(states[i] >> (8 * k));
}

unsigned char* readByteData_Yafan(char* srcFilePath, size_t* byteLength, int* status)
{
    return read_all(srcFilePath, byteLength, status);
}

uint16_t* readUInt16Data_systemEndian_Yafan(char* p, size_t* n, int* s) { return read_values<uint16_t>(p, n, s, false); }
uint16_t* readUInt16Data_Yafan(char* p, size_t* n, int* s) { return read_values<uint16_t>(p, n, s, !host_is_little_endian()); }
uint32_t* readUInt32Data_systemEndian_Yafan(char* p, size_t* n, int* s) { return read_values<uint32_t>(p, n, s, false); }
uint32_t* readUInt32Data_Yafan(char* p, size_t* n, int* s) { return read_values<uint32_t>(p, n, s, !host_is_little_endian()); }
float* readFloatData_systemEndian_Yafan(char* p, size_t* n, int* s) { return read_values<float>(p, n, s, false); }
float* readFloatData_Yafan(char* p, size_t* n, int* s) { return read_values<float>(p, n, s, !host_is_little_endian()); }
double* readDoubleData_systemEndian_Yafan(char* p, size_t* n, int* s) { return read_values<double>(p, n, s, false); }
double* readDoubleData_Yafan(char* p, size_t* n, int* s) { return read_values<double>(p, n, s, !host_is_little_endian()); }

void writeByteData_Yafan(unsigned char* bytes, size_t byteLength, char* tgtFilePath, int* status)
{
    write_all(bytes, byteLength, tgtFilePath, status);
}

void writeUShortData_inBytes_Yafan(unsigned short* states, size_t stateLength, char* tgtFilePath, int* status)
{
    write_values_le(states, stateLength, tgtFilePath, status);
}

void writeUIntData_inBytes_Yafan(unsigned int* states, size_t stateLength, char* tgtFilePath, int* status)
{
    write_values_le(states, stateLength, tgtFilePath, status);
}

void writeFloatData_inBytes_Yafan(float* data, size_t nbEle, char* tgtFilePath, int* status)
{
    write_values_le(data, nbEle, tgtFilePath, status);
}

void writeDoubleData_inBytes_Yafan(double* data, size_t nbEle, char* tgtFilePath, int* status)
{
    write_values_le(data, nbEle, tgtFilePath, status);
}
