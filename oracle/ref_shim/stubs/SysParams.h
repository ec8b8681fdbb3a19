#pragma once
namespace medyan {
struct MechParamsStub { int cylThresh = 0; };
struct SysParams {
    static const MechParamsStub& Mechanics() { static MechParamsStub m; return m; }
};
}
