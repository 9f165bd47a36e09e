#ifndef CUSZP_INCLUDE_CUSZP_CUSZP_TIMER_H
#define CUSZP_INCLUDE_CUSZP_CUSZP_TIMER_H

// CUDA-event timer on the legacy default stream; same class layout and members
// as the reference's include/cuSZp/cuSZp_timer.h:7-23 (replaces src/cuSZp_timer.cu).
// The events are created once per timer and released by the destructor.

#include <cuda.h>
#include <cuda_runtime.h>

struct PrivateTimingGPU {
    cudaEvent_t start;
    cudaEvent_t stop;
};

class TimingGPU
{
    private:
        PrivateTimingGPU *privateTimingGPU;

    public:
        TimingGPU();
        ~TimingGPU();
        void StartCounter();
        void StartCounterFlags();
        float GetCounter();

};

#endif // CUSZP_INCLUDE_CUSZP_CUSZP_TIMER_H
