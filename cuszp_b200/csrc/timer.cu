// timer.cu -- TimingGPU (include/cuSZp/cuSZp_timer.h): CUDA events recorded on
// the legacy default stream, as the reference's src/cuSZp_timer.cu:12-41 does,
// but created once per timer and destroyed with it.
#include "../../include/cuSZp/cuSZp_timer.h"

TimingGPU::TimingGPU()
{
    privateTimingGPU = new PrivateTimingGPU;
    cudaEventCreate(&privateTimingGPU->start);
    cudaEventCreate(&privateTimingGPU->stop);
}

TimingGPU::~TimingGPU()
{
    cudaEventDestroy(privateTimingGPU->start);
    cudaEventDestroy(privateTimingGPU->stop);
    delete privateTimingGPU;
}

void TimingGPU::StartCounter()
{
    cudaEventRecord(privateTimingGPU->start, 0);
}

void TimingGPU::StartCounterFlags()
{
    // blocking-sync events: the host thread sleeps in GetCounter instead of spinning
    cudaEventDestroy(privateTimingGPU->start);
    cudaEventDestroy(privateTimingGPU->stop);
    cudaEventCreateWithFlags(&privateTimingGPU->start, cudaEventBlockingSync);
    cudaEventCreateWithFlags(&privateTimingGPU->stop, cudaEventBlockingSync);
    cudaEventRecord(privateTimingGPU->start, 0);
}

float TimingGPU::GetCounter()
{
    float ms = 0.0f;
    cudaEventRecord(privateTimingGPU->stop, 0);
    cudaEventSynchronize(privateTimingGPU->stop);
    cudaEventElapsedTime(&ms, privateTimingGPU->start, privateTimingGPU->stop);
    return ms;
}
