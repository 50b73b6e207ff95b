// Test infrastructure: builds the B200ComputeBackend drop-in class against the
// reference's own IComputeBackend.h (proving it overrides every pure virtual
// with the reference's exact signatures), links it to libimage360_b200.so and
// exercises the calls that need no GPU.  Exit code 0 on success.
#include "image360_b200_backend.hpp"

#include <cstdio>
#include <cstring>
#include <memory>

using namespace WindowsApp::Compute;

int main()
{
    std::shared_ptr<IComputeBackend> backend = std::make_shared<B200ComputeBackend>();
    unsigned short data[4] = {100, 200, 300, 400};
    // Before Initialize: CUDA_ERROR "Not initialized." (CpuComputeBackend.cpp:117 convention).
    if (backend->ApplyGain(data, 4, 2.0f) != ComputeResult::CUDA_ERROR) return 1;
    if (std::strcmp(backend->GetLastError(), "Not initialized.") != 0) return 2;
    if (backend->BlockMatchAlign(nullptr, nullptr, 0, 0, 0, 0, nullptr, 0, 0) != ComputeResult::NOT_SUPPORTED) return 3;
    if (std::strstr(backend->GetLastError(), "not supported") == nullptr) return 4;
    auto* ext = dynamic_cast<IRenderBlendBackend*>(backend.get());
    if (!ext) return 5;
    ComputeResult r = backend->Initialize();
    std::printf("initialize=%d gpu=%d msg=%s\n", static_cast<int>(r), backend->IsInitialized() ? 1 : 0, backend->GetLastError());
    if (r == ComputeResult::SUCCESS)
    {
        if (backend->ApplyGain(data, 4, 2.0f) != ComputeResult::SUCCESS) return 6;
        if (data[0] != 200 || data[3] != 800) return 7;
        backend->Shutdown();
    }
    else if (r != ComputeResult::NO_GPU)
        return 8;
    return 0;
}
