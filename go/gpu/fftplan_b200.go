//  FFT plan "B200" for hotspin's FFTInterface registry: the FP64 3-D real FFT of libhsb200.so
//  (hsb_fft_plan_*, include/hotspin_b200.h) with the semantics of FFTPlanX (gpu/fftplanX.go),
//  selected with -fft=B200 (gpu/fftinterface.go:16-42, frontend/main.go).  Drop into
//  src/hotspin-core/gpu/ beside fftplanX.go, with hsb200.go for the cgo flags.  Not compiled in
//  this repository: no Go toolchain here.

package gpu

/*
#include "hotspin_b200.h"
*/
import "C"

import (
	"unsafe"

	. "hotspin-core/common"
)

func init() {
	fftPlans["B200"] = NewFFTPlanB200
}

// FFTPlanB200 keeps FFTPlanX's contract: Forward reads the data block and writes the padded
// spectrum (outputSize = logic size with two more doubles per row), Inverse reads a spectrum
// and writes the cropped real block.  Unlike FFTPlanX it needs no padding buffer from the
// caller and leaves Inverse's input spectrum unchanged.
type FFTPlanB200 struct {
	dataSize   [3]int
	logicSize  [3]int
	outputSize [3]int
	plan       C.hsb_fft_plan
	Stream
}

func NewFFTPlanB200(dataSize, logicSize []int) FFTInterface {
	Assert(len(dataSize) == 3)
	Assert(len(logicSize) == 3)
	fft := new(FFTPlanB200)
	outputSize := FFTOutputSize(logicSize)
	var d, l [3]C.int
	for i := range fft.dataSize {
		fft.dataSize[i], fft.logicSize[i], fft.outputSize[i] = dataSize[i], logicSize[i], outputSize[i]
		d[i], l[i] = C.int(dataSize[i]), C.int(logicSize[i])
	}
	fft.Stream = NewStream()
	if rc := C.hsb_fft_plan_create(&d[0], &l[0], unsafe.Pointer(uintptr(fft.Stream)), &fft.plan); rc != 0 {
		panic(InputErr("FFT plan B200: " + C.GoString(C.hsb_last_error())))
	}
	return fft
}

func (fft *FFTPlanB200) Forward(in, out *Array) {
	AssertMsg(in.size4D[0] == 1, "1")
	AssertMsg(out.size4D[0] == 1, "2")
	CheckSize(in.size3D, fft.dataSize[:])
	CheckSize(out.size3D, fft.outputSize[:])
	src := (*C.double)(unsafe.Pointer(uintptr(in.Pointer())))
	dst := (*C.double)(unsafe.Pointer(uintptr(out.Pointer())))
	if rc := C.hsb_fft_forward(fft.plan, src, dst); rc != 0 {
		panic(InputErr("FFT plan B200 forward: " + C.GoString(C.hsb_last_error())))
	}
}

func (fft *FFTPlanB200) Inverse(in, out *Array) {
	CheckSize(in.size3D, fft.outputSize[:])
	CheckSize(out.size3D, fft.dataSize[:])
	src := (*C.double)(unsafe.Pointer(uintptr(in.Pointer())))
	dst := (*C.double)(unsafe.Pointer(uintptr(out.Pointer())))
	if rc := C.hsb_fft_inverse(fft.plan, src, dst); rc != 0 {
		panic(InputErr("FFT plan B200 inverse: " + C.GoString(C.hsb_last_error())))
	}
}

func (fft *FFTPlanB200) Free() {
	if fft.plan != nil {
		C.hsb_fft_plan_destroy(fft.plan)
		fft.plan = nil
	}
}
