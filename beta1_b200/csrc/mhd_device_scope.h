// Device binding of a context's entry points.
//
// A context lives on the device that was current when it was created.  Every
// entry point that touches it makes that device current for the duration of
// the call and puts the caller's device back on return, so a process that
// holds contexts on several GPUs may call any of them from any current
// device.  Api supplies get(int *) / set(int) returning 0 on success (the CUDA
// runtime in the library, a fake in the host test of this bookkeeping).
#ifndef MHD_DEVICE_SCOPE_H
#define MHD_DEVICE_SCOPE_H

template <class Api>
class DeviceScope
{
  public:
    // want < 0: no device to bind (null context); nothing is changed
    explicit DeviceScope(int want)
    {
        if (want < 0)
            return;
        int cur = -1;
        if (Api::get(&cur) != 0)
        {
            ok_ = false;
            return;
        }
        if (cur == want)
            return;
        if (Api::set(want) != 0)
        {
            ok_ = false;
            return;
        }
        prev_ = cur;
    }
    ~DeviceScope()
    {
        if (prev_ >= 0)
            Api::set(prev_);
    }
    DeviceScope(const DeviceScope &) = delete;
    DeviceScope &operator=(const DeviceScope &) = delete;
    // false when the context's device could not be made current
    bool ok() const { return ok_; }

  private:
    int prev_ = -1; // caller's device to restore, -1 if unchanged
    bool ok_ = true;
};

#endif
